"""GPU parity of the fused FP32 column-forward kernels against the FP64 oracle.

The oracle runs the reference sequence (gas optics -> cloud optics -> add_to -> solver ->
broadband reduction -> heating rate) in FP64; the fused kernels run the same physics in FP32
with compensated g-point sums.  Bounds: broadband fluxes within 5e-3 W/m2 of FP64 and heating
rates within 0.01 K/day at every layer, including the ~0.1 Pa-thick top layers (the targets
stated for the FP32 product are 0.05 W/m2 and 0.01 K/day).  The fused kernels form heating
rates from per-layer flux divergence, not from differences of FP32 level fluxes.
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

pytestmark = pytest.mark.gpu
HR_TOL = 0.01


def _solvers(tables):
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    return base, Fused_solver(base)


def _check(got, ref, atm, what):
    for k in ("flux_up", "flux_dn", "flux_net"):
        err = np.max(np.abs(got[k].double().cpu().numpy() - ref[k]))
        assert err < 5e-3, f"{what} {k}: max abs err {err:.3e} W/m2"
    hr = got["heating_rate"].double().cpu().numpy()
    href = ref["heating_rate"]
    e = np.abs(hr - href)
    assert np.max(e) < HR_TOL, f"{what} heating rate: {np.max(e):.3e} K/day"


@pytest.mark.parametrize("nlay", [23, 60, 128])
@pytest.mark.parametrize("clouds", [False, True])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("chunk", [8, 16])
def test_fused_lw_matches_oracle(oracle_mod, tables, gpu, nlay, clouds, top_at_1, chunk):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    if chunk == 8 and nlay > 128:
        pytest.skip("chunk 8 covers at most 128 layers")
    base, fused = _solvers(tables)
    fused.chunk = chunk
    atm = S.make_atmosphere(37, nlay, seed=50 + nlay, clouds=clouds, top_at_1=top_at_1)
    ref = oracle_mod.forward_lw(oracle_mod.GasOptics(tables["lw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_lw"]) if clouds else None, atm)
    got = fused.solve_lw(atm_to_device(atm, torch.float32, gpu), with_clouds=clouds)
    torch.cuda.synchronize()
    _check(got, ref, atm, f"lw nlay={nlay} clouds={clouds} top_at_1={top_at_1} chunk={chunk}")


def test_fused_lw_matches_staged_fp32(tables, gpu):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = atm_to_device(S.make_atmosphere(300, 64, seed=9, clouds=True), torch.float32, gpu)
    a = fused.solve_lw(atm)
    b = base.solve_lw(atm)
    for k in ("flux_up", "flux_dn"):
        assert float((a[k] - b[k]).abs().max()) < 5e-3


def _vary_surface(atm, seed):
    """Per-band albedos with direct != diffuse and a non-unit TSI scaling."""
    rng = np.random.default_rng(seed)
    ncol, nb = atm["sfc_alb_dir"].shape
    atm["sfc_alb_dir"] = rng.uniform(0.02, 0.9, (ncol, nb))
    atm["sfc_alb_dif"] = rng.uniform(0.02, 0.9, (ncol, nb))
    atm["tsi_scaling"] = rng.uniform(0.9, 1.1, ncol)
    return atm


def _check_sw(got, ref, what):
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net"):
        err = np.max(np.abs(got[k].double().cpu().numpy() - ref[k]))
        assert err < 5e-3, f"{what} {k}: max abs err {err:.3e} W/m2"
    e = np.abs(got["heating_rate"].double().cpu().numpy() - ref["heating_rate"])
    assert np.max(e) < HR_TOL, f"{what} heating rate: {np.max(e):.3e} K/day"


@pytest.mark.parametrize("nlay", [23, 60, 128])
@pytest.mark.parametrize("clouds", [False, True])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("chunk", [8, 16])
def test_fused_sw_matches_oracle(oracle_mod, tables, gpu, nlay, clouds, top_at_1, chunk):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    fused.chunk = chunk
    atm = _vary_surface(S.make_atmosphere(37, nlay, seed=70 + nlay, clouds=clouds, top_at_1=top_at_1), nlay)
    ref = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]) if clouds else None, atm)
    got = fused.solve_sw(atm_to_device(atm, torch.float32, gpu), with_clouds=clouds)
    torch.cuda.synchronize()
    _check_sw(got, ref, f"sw nlay={nlay} clouds={clouds} top_at_1={top_at_1} chunk={chunk}")


def test_fused_sw_low_sun_and_resonance(oracle_mod, tables, gpu):
    """mu0 over [0.02, 1] including values where k mu0 = 1 for purely absorbing g-points
    (k = 2 at w0 = 0, i.e. mu0 = 0.5): exercises the factored k mu0 = 1 expressions of the FP32
    two-stream and its thick-layer branch, in the fused kernel and in the per-stage FP32 solver
    (fluxes; its heating rates come from FP32 level-flux differences)."""
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = _vary_surface(S.make_atmosphere(64, 60, seed=5, clouds=True), 3)
    atm["mu0"] = np.concatenate([np.linspace(0.02, 1.0, 48), 0.5 + np.linspace(-1e-3, 1e-3, 16)])
    ref = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]), atm)
    got = fused.solve_sw(atm_to_device(atm, torch.float32, gpu))
    torch.cuda.synchronize()
    _check_sw(got, ref, "sw low sun / resonance")
    staged = base.solve_sw(atm_to_device(atm, torch.float32, gpu))
    torch.cuda.synchronize()
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net"):
        e = np.max(np.abs(staged[k].double().cpu().numpy() - ref[k]))
        assert e < 5e-3, f"staged sw low sun / resonance {k}: {e:.3e} W/m2"


def test_fused_sw_matches_staged_fp32(tables, gpu):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = atm_to_device(_vary_surface(S.make_atmosphere(300, 64, seed=9, clouds=True), 1), torch.float32, gpu)
    a = fused.solve_sw(atm)
    b = base.solve_sw(atm)
    for k in ("flux_up", "flux_dn", "flux_dn_dir"):
        assert float((a[k] - b[k]).abs().max()) < 5e-3


@pytest.mark.parametrize("ncol,nlay", [(1, 2), (2, 3), (1, 9), (5, 17)])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_fused_small_domains_match_oracle(oracle_mod, tables, gpu, ncol, nlay, top_at_1):
    """Domains far below one warp of columns and one chunk of layers (a single CTA with one
    warp, most lanes and chunk layers idle) for both fused kernels at both chunk lengths."""
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = _vary_surface(S.make_atmosphere(ncol, nlay, seed=90 + nlay, clouds=True, top_at_1=top_at_1), nlay)
    ref_lw = oracle_mod.forward_lw(oracle_mod.GasOptics(tables["lw"], S.ATM_GASES),
                                   oracle_mod.CloudOptics(tables["cloud_lw"]), atm)
    ref_sw = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                   oracle_mod.CloudOptics(tables["cloud_sw"]), atm)
    dev = atm_to_device(atm, torch.float32, gpu)
    for chunk in (8, 16):
        fused.chunk = chunk
        got = fused.solve_lw(dev, with_clouds=True)
        torch.cuda.synchronize()
        _check(got, ref_lw, atm, f"lw ncol={ncol} nlay={nlay} chunk={chunk}")
        got = fused.solve_sw(dev, with_clouds=True)
        torch.cuda.synchronize()
        _check_sw(got, ref_sw, f"sw ncol={ncol} nlay={nlay} chunk={chunk}")


def test_fused_forward_from_two_host_threads(tables, gpu):
    """The fused entry points are called from two host threads at once, each on its own
    stream with its own output buffers and the same k-distribution handles (handles are
    immutable after creation; the launchers' one-time per-device set-up is locked).  Every
    result equals the single-thread result bit for bit."""
    import threading

    import torch
    from rrtmgp_b200.solver import Fused_solver, atm_to_device
    base, fused = _solvers(tables)
    atms = [atm_to_device(S.make_atmosphere(64, 60 + 30 * i, seed=70 + i, clouds=True), torch.float32, gpu)
            for i in range(2)]
    want = []
    for a in atms:
        lw, sw = fused.solve_lw(a), fused.solve_sw(a)
        want.append({**{"lw_" + k: v.clone() for k, v in lw.items()}, **{"sw_" + k: v.clone() for k, v in sw.items()}})
    torch.cuda.synchronize()
    got, errors = [None, None], []

    def run(i):
        try:
            f = Fused_solver(base)
            s = torch.cuda.Stream(device=gpu)
            with torch.cuda.stream(s):
                for _ in range(20):
                    lw, sw = f.solve_lw(atms[i]), f.solve_sw(atms[i])
                got[i] = {**{"lw_" + k: v.clone() for k, v in lw.items()},
                          **{"sw_" + k: v.clone() for k, v in sw.items()}}
            s.synchronize()
        except Exception as e:   # reported in the main thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=120)
    assert not errors, errors
    for i in range(2):
        for k, v in want[i].items():
            assert torch.equal(got[i][k], v), f"thread {i} {k}"


@pytest.mark.parametrize("top_at_1", [True, False])
def test_staged_fp32_heating_rates_match_oracle(oracle_mod, tables, gpu, top_at_1):
    """The per-stage FP32 path (class API sequence) forms heating rates from per-layer absorbed
    flux (rrtmgp_b200_heating_rate_{lw,sw}_layers_f32): within 0.01 K/day of FP64 at every
    layer, the ~0.1 Pa top layers included, where differences of its FP32 level fluxes are off
    by ~1 K/day."""
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, _ = _solvers(tables)
    atm = _vary_surface(S.make_atmosphere(37, 128, seed=61, clouds=True, top_at_1=top_at_1), 62)
    d = atm_to_device(atm, torch.float32, gpu)
    lw, sw = base.solve_lw(d, top_at_1=top_at_1), base.solve_sw(d, top_at_1=top_at_1)
    torch.cuda.synchronize()
    rlw = oracle_mod.forward_lw(oracle_mod.GasOptics(tables["lw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_lw"]), atm)
    rsw = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]), atm)
    _check(lw, rlw, atm, f"staged fp32 lw top_at_1={top_at_1}")
    _check_sw(sw, rsw, f"staged fp32 sw top_at_1={top_at_1}")


@pytest.mark.parametrize("nlay,top_at_1", [(300, True), (520, False), (1000, True)])
def test_fused_deep_columns_on_clusters(oracle_mod, tables, gpu, nlay, top_at_1):
    """Columns of more than 16 chunks (here 19 to 63 chunks of 16 layers) run on a thread-block
    cluster of 2 to 4 CTAs per column, the chunk maps in distributed shared memory; LW and SW
    against the oracle with the bounds of the other fused tests."""
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = _vary_surface(S.make_atmosphere(9, nlay, seed=nlay, clouds=True, top_at_1=top_at_1), nlay + 1)
    d = atm_to_device(atm, torch.float32, gpu)
    lw, sw = fused.solve_lw(d), fused.solve_sw(d)
    torch.cuda.synchronize()
    rlw = oracle_mod.forward_lw(oracle_mod.GasOptics(tables["lw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_lw"]), atm)
    rsw = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]), atm)
    _check(lw, rlw, atm, f"deep lw nlay={nlay}")
    _check_sw(sw, rsw, f"deep sw nlay={nlay}")
