"""Aerosol optics (Aerosol_optics_gpu, src_cuda/Aerosol_optics.cu): oracle checks on the CPU and
GPU parity of the FP64 and FP32 kernels against the oracle."""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S


def _case(ncol=7, nlay=9, top_at_1=True, seed=3):
    atm = S.make_atmosphere(ncol, nlay, seed=seed, clouds=False, top_at_1=top_at_1)
    aer, rh = S.make_aerosols(atm["play"], seed=seed + 1)
    return atm, aer, rh


def test_oracle_aerosol_by_hand(oracle_mod):
    """One species at a time against a direct numpy evaluation of the table look-up."""
    t = S.make_aerosol_luts()
    atm, aer, rh = _case()
    plev = atm["plev"]
    dpg = np.abs(plev[:-1] - plev[1:]) / 9.81
    ihum = np.minimum(np.searchsorted(t["relative_humidity2"], rh, side="left"), len(t["relative_humidity2"]) - 1)
    # name -> (hydrophilic?, 0-based type), as in the reference kernel
    spec = {"aermr01": (1, 0), "aermr02": (1, 1), "aermr03": (1, 2), "aermr04": (0, 0), "aermr05": (0, 7),
            "aermr06": (0, 5), "aermr07": (1, 3), "aermr08": (0, 9), "aermr09": (0, 10), "aermr10": (0, 10),
            "aermr11": (1, 4)}
    zero = {k: np.zeros_like(v) for k, v in aer.items()}
    for name, (phil, typ) in spec.items():
        one = dict(zero)
        one[name] = aer[name]
        out = oracle_mod.aerosol_optics(t, one, rh, plev)
        for b in (0, 5, 13):
            if phil:
                me = t["mass_ext_sw_hydrophilic"][typ][ihum, b]
                sa = t["ssa_sw_hydrophilic"][typ][ihum, b]
                ga = t["asymmetry_sw_hydrophilic"][typ][ihum, b]
            else:
                me = t["mass_ext_sw_hydrophobic"][typ, b]
                sa = t["ssa_sw_hydrophobic"][typ, b]
                ga = t["asymmetry_sw_hydrophobic"][typ, b]
            tau = aer[name] * dpg * me
            eps = np.finfo(np.float64).eps
            ts = tau * sa
            np.testing.assert_allclose(out["tau"][b], tau, rtol=1e-13)
            np.testing.assert_allclose(out["ssa"][b], ts / np.maximum(tau, eps), rtol=1e-12)
            np.testing.assert_allclose(out["g"][b], ts * ga / np.maximum(ts, eps), rtol=1e-12)


def test_oracle_aerosol_zero_and_clamp(oracle_mod):
    t = S.make_aerosol_luts()
    atm, aer, rh = _case()
    zero = {k: np.zeros_like(v) for k, v in aer.items()}
    out = oracle_mod.aerosol_optics(t, zero, rh, atm["plev"])
    assert not out["tau"].any() and not out["ssa"].any() and not out["g"].any()
    # rh above the table's last class uses the last class
    hi = oracle_mod.aerosol_optics(t, aer, np.full_like(rh, 1.5), atm["plev"])
    top = oracle_mod.aerosol_optics(t, aer, np.full_like(rh, 1.0), atm["plev"])
    np.testing.assert_array_equal(hi["tau"], top["tau"])
    # orientation: |dp| gives the same optics for a flipped column
    atm2, aer2, rh2 = _case(top_at_1=False)
    a = oracle_mod.aerosol_optics(t, aer, rh, atm["plev"])
    b = oracle_mod.aerosol_optics(t, {k: v[::-1].copy() for k, v in aer.items()}, rh[::-1].copy(),
                                  atm["plev"][::-1].copy())
    np.testing.assert_allclose(a["tau"], b["tau"][:, ::-1], rtol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("profile", [False, True])
def test_aerosol_gpu_matches_oracle(oracle_mod, gpu, dtype, profile):
    import torch
    from rrtmgp_b200 import api
    t = S.make_aerosol_luts()
    atm, aer, rh = _case(ncol=33, nlay=20)
    if profile:   # (nlay,) profiles and one scalar broadcast over the columns
        aer = {k: (v[:, 0].copy() if i % 2 else v) for i, (k, v) in enumerate(aer.items())}
        aer["aermr05"] = np.array([3e-9])
    ref = oracle_mod.aerosol_optics(t, aer, rh, atm["plev"])
    dt = getattr(torch, dtype)
    ao = api.Aerosol_optics(t)
    d = {k: torch.as_tensor(np.ascontiguousarray(v), dtype=dt, device=gpu) for k, v in aer.items()}
    got = ao.aerosol_optics(d, torch.as_tensor(rh, dtype=dt, device=gpu),
                            torch.as_tensor(atm["plev"], dtype=dt, device=gpu))
    torch.cuda.synchronize()
    rtol = 1e-13 if dtype == "float64" else 2e-6
    # ssa and g divide by max(tau, eps) and max(tau ssa, eps) with the precision's epsilon
    # (as the reference builds): FP32 is compared where those do not bind
    feps = np.finfo(np.float32).eps
    masks = {"tau": np.ones(ref["tau"].shape, bool), "ssa": ref["tau"] > 2 * feps,
             "g": ref["tau"] * ref["ssa"] > 2 * feps}
    for k in ("tau", "ssa", "g"):
        g = got[k].double().cpu().numpy()
        m = masks[k] if dtype == "float32" else masks["tau"]
        assert m.any()
        np.testing.assert_allclose(g[m], ref[k][m], rtol=rtol, atol=1e-30, err_msg=k)


@pytest.mark.gpu
def test_aerosol_missing_species(gpu):
    import torch
    from rrtmgp_b200 import _abi, api
    t = S.make_aerosol_luts()
    atm, aer, rh = _case()
    aer.pop("aermr07")
    ao = api.Aerosol_optics(t)
    d = {k: torch.as_tensor(v, device=gpu) for k, v in aer.items()}
    with pytest.raises(_abi.RrtmgpError) as e:
        ao.aerosol_optics(d, torch.as_tensor(rh, device=gpu), torch.as_tensor(atm["plev"], device=gpu))
    assert e.value.status == _abi.ERR_MISSING_GAS


@pytest.mark.gpu
@pytest.mark.parametrize("delta_aerosol", [False, True])
def test_solve_sw_with_aerosols(oracle_mod, tables, gpu, delta_aerosol):
    """Radiation_solver.solve_sw (FP64 staged path) with clouds and aerosols added by band,
    against the oracle's solve_gpu sequence."""
    import torch
    from rrtmgp_b200.solver import Radiation_solver, atm_to_device
    tab = S.make_aerosol_luts()
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES,
                            aerosol_sw=tab, delta_aerosol=delta_aerosol)
    atm = S.make_atmosphere(9, 30, seed=81, clouds=True)
    atm["aerosols"], atm["rh"] = S.make_aerosols(atm["play"], seed=82)
    d = atm_to_device(atm, torch.float64, gpu)
    d["aerosols"] = {k: torch.as_tensor(v, dtype=torch.float64, device=gpu) for k, v in atm["aerosols"].items()}
    d["rh"] = torch.as_tensor(atm["rh"], dtype=torch.float64, device=gpu)
    got = {k: v.clone() for k, v in base.solve_sw(d, with_aerosols=True).items()}
    plain = {k: v.clone() for k, v in base.solve_sw(d).items()}
    torch.cuda.synchronize()
    ref = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]), atm, aerosol_tables=tab,
                                delta_aerosol=delta_aerosol)
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate"):
        g = got[k].double().cpu().numpy()
        # heating rates difference level fluxes over ~0.1 Pa layers: 1e-6 K/day absolute
        np.testing.assert_allclose(g, ref[k], rtol=1e-8, atol=1e-6 if k == "heating_rate" else 1e-8, err_msg=k)
    # the aerosols change the fluxes
    assert float((plain["flux_dn_dir"] - got["flux_dn_dir"]).abs().max()) > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("delta_aerosol", [False, True])
@pytest.mark.parametrize("top_at_1,nlay", [(True, 60), (False, 128), (True, 200)])
def test_fused_sw_with_aerosols(oracle_mod, tables, gpu, delta_aerosol, top_at_1, nlay):
    """The fused FP32 shortwave kernel with aerosols (rrtmgp_b200_forward_sw_aer_f32): aerosol
    optics per (layer, band) inside the kernel, delta-scaled or not, added after the clouds;
    against the oracle's solve_gpu sequence with the fused kernels' bounds (5e-3 W/m2,
    0.01 K/day), profiles and a scalar among the species."""
    import torch
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    tab = S.make_aerosol_luts()
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES,
                            aerosol_sw=tab, delta_aerosol=delta_aerosol)
    atm = S.make_atmosphere(37, nlay, seed=83 + nlay, clouds=True, top_at_1=top_at_1)
    aer, rh = S.make_aerosols(atm["play"], seed=84)
    aer["aermr02"] = aer["aermr02"][:, 0].copy()   # a profile
    aer["aermr07"] = np.array([2e-9])               # a scalar
    atm["aerosols"], atm["rh"] = aer, rh
    d = atm_to_device(atm, torch.float32, gpu)
    d["aerosols"] = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous() for k, v in aer.items()}
    d["rh"] = torch.as_tensor(rh, dtype=torch.float32, device=gpu).contiguous()
    fused = Fused_solver(base)
    got = {k: v.clone() for k, v in fused.solve_sw(d, with_aerosols=True).items()}
    plain = {k: v.clone() for k, v in fused.solve_sw(d).items()}
    torch.cuda.synchronize()
    ref = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]), atm, aerosol_tables=tab,
                                delta_aerosol=delta_aerosol)
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate"):
        e = float(np.max(np.abs(got[k].double().cpu().numpy() - ref[k])))
        assert e < (0.01 if k == "heating_rate" else 5e-3), f"{k}: {e:.3e}"
    assert float((plain["flux_dn_dir"] - got["flux_dn_dir"]).abs().max()) > 1e-3


@pytest.mark.gpu
def test_sw_adjoint_with_aerosols_matches_fd(oracle_mod, tables, gpu):
    """SW forward + adjoint with aerosols in the recomputed forward
    (rrtmgp_b200_forward_adjoint_sw_aer_f32): gradients against FP64 central differences of the
    oracle's sequence with the same aerosols (bounds of the other adjoint tests), fluxes against
    its forward."""
    import torch
    from test_gpu_adjoint import _check, _fd, _fd_bands, _get, _informative, _sw_seeds
    from rrtmgp_b200.autodiff import adjoint_sw
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    tab = S.make_aerosol_luts()
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES,
                            aerosol_sw=tab, delta_aerosol=True)
    ncol, nlay = 3, 24
    atm = S.make_atmosphere(ncol, nlay, seed=85, clouds=True)
    atm["mu0"] = np.array([0.3, 0.6, 0.9])
    atm["aerosols"], atm["rh"] = S.make_aerosols(atm["play"], seed=86)
    kd, cl = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES), oracle_mod.CloudOptics(tables["cloud_sw"])
    fwd = lambda a: oracle_mod.forward_sw(kd, cl, a, aerosol_tables=tab, delta_aerosol=True)  # noqa: E731
    seeds = _sw_seeds(nlay, ncol, np.random.default_rng(87))
    d = atm_to_device(atm, torch.float32, gpu)
    d["aerosols"] = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous()
                     for k, v in atm["aerosols"].items()}
    d["rh"] = torch.as_tensor(atm["rh"], dtype=torch.float32, device=gpu).contiguous()
    t = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous() for k, v in seeds.items()}
    fl, g = adjoint_sw(Fused_solver(base), d, t["flux_up"], t["flux_dn"], t["flux_dn_dir"], t["heating_rate"],
                       with_fluxes=True, with_aerosols=True)
    torch.cuda.synchronize()
    ref = fwd(atm)
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "heating_rate"):
        e = float(np.max(np.abs(fl[k].double().cpu().numpy() - ref[k])))
        assert e < (0.01 if k == "heating_rate" else 5e-3), f"{k}: {e:.3e}"
    got = {k: v.double().cpu().numpy() for k, v in g.items()}
    for key in ("tlay", "h2o", "o3"):
        _check(f"sw+aerosol d/d{key}", got[key], _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))
    _check("sw+aerosol d/dsfc_alb_dif", got["sfc_alb_dif"], _fd_bands(fwd, atm, seeds, "sfc_alb_dif"))
    if (atm["lwp"] > 0).any():
        _check("sw+aerosol d/dlwp", got["lwp"], _fd(fwd, atm, seeds, "lwp"), atm["lwp"] > 0)
