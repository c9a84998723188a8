"""Batched forward of uneven grids in one persistent launch (rrtmgp_b200_batch_*).

Parity: with the per-grid chunk rule (longwave 16 layers per warp; shortwave 8 up to 128
layers, else 16) the batched
results equal the per-grid fused launches to FP32 rounding (the same per-column code, compiled
in another kernel, may contract multiply-adds differently: SAME_TOL), whatever the number of
columns per CTA; the persistent launch and its graph replay agree bit for bit; every tile
shape the autotuner may pick matches the FP64 oracle within the fused kernels' bounds
(5e-3 W/m2, 0.01 K/day).  Graph replays read the inputs in place.
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

HR_TOL = 0.01
FLUX_TOL = 5e-3
SAME_TOL = 2e-3     # W/m2 and K/day: same algorithm and chunk length, FP32 rounding only

# (ncol, nlay, clouds, top_at_1): uneven shapes, both orientations, single columns, the
# smallest and largest layer counts, clear and cloudy grids in one batch.
GRIDS = [(37, 23, True, True), (64, 60, False, True), (5, 128, True, False), (1, 3, True, True),
         (70, 129, True, True), (33, 200, True, False), (9, 256, True, True), (300, 41, True, True)]


def _base(tables):
    from rrtmgp_b200.solver import Radiation_solver
    return Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)


def _atms(gpu, grids=GRIDS, seed=0):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    host, dev = [], []
    for i, (ncol, nlay, clouds, top) in enumerate(grids):
        a = S.make_atmosphere(ncol, nlay, seed=seed + 100 + i, clouds=clouds, top_at_1=top)
        rng = np.random.default_rng(seed + i)
        a["sfc_alb_dif"] = rng.uniform(0.02, 0.9, a["sfc_alb_dif"].shape)
        a["tsi_scaling"] = rng.uniform(0.9, 1.1, ncol)
        d = atm_to_device(a, torch.float32, gpu)
        if not clouds:
            for k in ("lwp", "iwp", "rel", "rei"):
                d[k] = None
        host.append(a)
        dev.append(d)
    return host, dev


def _rule_plan(bf):
    """The per-grid chunk rule (longwave 16; shortwave 8 up to 128 layers, else 16) with the most
    columns per CTA that fit."""
    for d in bf.domains():
        for b in bf.bins():
            cl = 16 if d == 0 else (8 if b <= 16 else 16)
            w = -(-8 * b // cl)
            for p in range(min(16 // w, 15), 0, -1):
                try:
                    bf.set_plan(d, b, cl, p)
                    break
                except Exception:
                    continue


def _copy(out):
    return [{dom: {k: v.clone() for k, v in o[dom].items()} for dom in o} for o in out]


def _same(a, b, what):
    import torch
    assert torch.isfinite(a).all(), what
    d = float((a - b).abs().max())
    assert d <= SAME_TOL, f"{what}: {d:.3e}"


@pytest.mark.gpu
def test_batch_persistent_and_graph_equal_per_grid(tables, gpu):
    import torch
    from rrtmgp_b200.batch import Batched_forward
    base = _base(tables)
    _, atms = _atms(gpu)
    bf = Batched_forward(base, atms)
    _rule_plan(bf)
    ref = _copy(bf.run("per_grid"))
    first = None
    for mode in ("persistent", "graph", "graph"):
        for o in bf.out:
            for dom in o:
                for v in o[dom].values():
                    v.fill_(float("nan"))
        got = _copy(bf.run(mode))
        torch.cuda.synchronize()
        for i, (o, r) in enumerate(zip(got, ref)):
            for dom in r:
                for k in r[dom]:
                    _same(o[dom][k], r[dom][k], f"{mode} grid {i} {dom} {k}")
                    if first is not None:
                        assert torch.equal(o[dom][k], first[i][dom][k]), f"{mode} grid {i} {dom} {k}"
        first = first or got
    st = bf.stats()
    assert st["launches_persistent"] == 1 and st["launches_per_grid"] == 2 * len(GRIDS)
    bf.close()


def _check_oracle(oracle_mod, tables, host, got, what):
    glw = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES)
    gsw = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    clw = oracle_mod.CloudOptics(tables["cloud_lw"])
    csw = oracle_mod.CloudOptics(tables["cloud_sw"])
    for i, (a, o) in enumerate(zip(host, got)):
        clouds = GRIDS[i][2]
        for dom, ref in (("lw", oracle_mod.forward_lw(glw, clw if clouds else None, a)),
                         ("sw", oracle_mod.forward_sw(gsw, csw if clouds else None, a))):
            for k in ref:
                if k not in o[dom]:
                    continue
                e = np.max(np.abs(o[dom][k].double().cpu().numpy() - ref[k]))
                tol = HR_TOL if k == "heating_rate" else FLUX_TOL
                assert e < tol, f"{what} grid {i} {dom} {k}: {e:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["heuristic", "chunk16", "one_column"])
def test_batch_tile_shapes_match_oracle(oracle_mod, tables, gpu, shape):
    import torch
    from rrtmgp_b200.batch import Batched_forward
    base = _base(tables)
    host, atms = _atms(gpu, seed=7)
    bf = Batched_forward(base, atms)
    for d in bf.domains():
        for b in bf.bins():
            if shape == "chunk16":
                bf.set_plan(d, b, 16, 1)
            elif shape == "one_column":
                bf.set_plan(d, b, 8 if b <= 16 else 16, 1)
    got = bf.run("graph")
    torch.cuda.synchronize()
    _check_oracle(oracle_mod, tables, host, got, shape)
    bf.close()


@pytest.mark.gpu
def test_batch_graph_replay_reads_inputs_in_place(tables, gpu):
    import torch
    from rrtmgp_b200.batch import Batched_forward
    base = _base(tables)
    _, atms = _atms(gpu, seed=3)
    bf = Batched_forward(base, atms)
    first = _copy(bf.run("graph"))
    for a in atms:
        a["tlay"].add_(1.5)
        a["mu0"].mul_(0.8)
    got = _copy(bf.run("graph"))
    _rule_plan(bf)
    again = _copy(bf.run("graph"))       # new plan: graph re-captured
    ref = _copy(bf.run("per_grid"))
    torch.cuda.synchronize()
    for i in range(len(atms)):
        assert not torch.equal(first[i]["lw"]["heating_rate"], got[i]["lw"]["heating_rate"])
        assert not torch.equal(first[i]["sw"]["flux_dn"], got[i]["sw"]["flux_dn"])
        for dom in ("lw", "sw"):
            for k in ref[i][dom]:
                _same(again[i][dom][k], ref[i][dom][k], f"grid {i} {dom} {k}")
                assert float((got[i][dom][k] - ref[i][dom][k]).abs().max()) < FLUX_TOL
    bf.close()


@pytest.mark.gpu
def test_batch_autotune_and_cache(tables, gpu, tmp_path):
    import torch
    from rrtmgp_b200.batch import Batched_forward, load_cache
    base = _base(tables)
    grids = [(400, 60, True, True), (150, 130, True, True), (64, 44, False, False)]
    _, atms = _atms(gpu, grids=grids, seed=11)
    bf = Batched_forward(base, atms)
    cache = tmp_path / "tiles.json"
    plan = bf.autotune(reps=1, cache=cache)
    entries = load_cache(cache)
    assert len(entries) == len(bf.domains()) * len(bf.bins())
    for (d, b), (cl, cols, us) in plan.items():
        assert cl in (8, 16) and 1 <= cols <= 15 and us > 0.0
        assert -(-8 * b // cl) * cols <= 16
    out = _copy(bf.run("graph"))
    bf2 = Batched_forward(base, atms)
    assert bf2.autotune(cache=cache) == plan   # from the cache, no timing
    out2 = bf2.run("persistent")
    torch.cuda.synchronize()
    for a, b in zip(out, out2):
        for dom in a:
            for k in a[dom]:
                assert torch.equal(a[dom][k], b[dom][k])
    bf.close()
    bf2.close()


@pytest.mark.gpu
def test_batch_single_domain(tables, gpu):
    import torch
    from rrtmgp_b200.batch import Batched_forward
    base = _base(tables)
    _, atms = _atms(gpu, grids=GRIDS[:4], seed=5)
    for lw, sw in ((True, False), (False, True)):
        bf = Batched_forward(base, atms, lw=lw, sw=sw)
        assert bf.domains() == ([0] if lw else [1])
        _rule_plan(bf)
        ref = _copy(bf.run("per_grid"))
        got = bf.run("persistent")
        torch.cuda.synchronize()
        for o, r in zip(got, ref):
            assert list(o) == (["lw"] if lw else ["sw"])
            for dom in r:
                for k in r[dom]:
                    _same(o[dom][k], r[dom][k], f"{dom} {k}")
        bf.close()


@pytest.mark.gpu
def test_batch_rejects_bad_plans(tables, gpu):
    from rrtmgp_b200 import _abi
    from rrtmgp_b200.batch import Batched_forward
    base = _base(tables)
    _, atms = _atms(gpu, grids=[(8, 200, True, True)], seed=2)
    bf = Batched_forward(base, atms)
    b = bf.bins()[0]
    for args in ((b, 12, 1), (b, 8, 1), (b, 16, 2), (0, 16, 1), (33, 16, 1)):
        with pytest.raises(_abi.RrtmgpError) as e:
            bf.set_plan(0, *args)
        assert e.value.status == _abi.ERR_ARG
    bf.close()


def test_batch_create_validates_on_host():
    """Argument checks run before any CUDA call (no GPU needed)."""
    import ctypes as C
    from rrtmgp_b200 import _abi
    from rrtmgp_b200.batch import BatchGrid
    lib = _abi.load()
    buf = C.c_void_p(16)     # never dereferenced: every case fails before reading arrays
    g = (BatchGrid * 1)()
    g[0].ncol, g[0].nlay = 4, 300
    g[0].play = g[0].plev = g[0].tlay = buf.value
    g[0].lw_flux_up = buf.value
    h = C.c_void_p()
    for nlay, msg in ((300, b"1 < nlay <= 256"), (1, b"1 < nlay <= 256"),
                      (40, b"longwave outputs without a longwave k-distribution")):
        g[0].nlay = nlay
        st = lib.rrtmgp_b200_batch_create(None, None, None, None, 1, C.cast(g, C.c_void_p), 1, C.byref(h))
        assert st == _abi.ERR_ARG and msg in lib.rrtmgp_b200_last_error()
        assert not h.value
    assert lib.rrtmgp_b200_batch_create(None, None, None, None, 1, None, 0, C.byref(h)) == _abi.ERR_ARG
    assert lib.rrtmgp_b200_batch_run(None, 0, None) == _abi.ERR_ARG
    assert lib.rrtmgp_b200_batch_destroy(None) == _abi.OK


def test_batch_cache_roundtrip(tmp_path):
    from rrtmgp_b200.batch import bins_of, cache_key, load_cache, save_cache
    assert bins_of([2, 8, 9, 40, 41, 256]) == [1, 2, 5, 6, 32]
    p = tmp_path / "t.json"
    save_cache(p, {cache_key("B200", 0, 256, 5): (8, 3, 41.5)})
    save_cache(p, {cache_key("B200", 1, 224, 25): (16, 1, 120.0)})
    c = load_cache(p)
    assert c == {"B200|lw|g256|bin5": (8, 3, 41.5), "B200|sw|g224|bin25": (16, 1, 120.0)}
