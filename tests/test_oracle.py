"""CPU tests of the FP64 oracle: analytic known answers and reference behaviours.

The oracle is the parity checker for the CUDA path, so it is itself pinned here against
closed-form solutions of the radiative transfer equations and against the invariants of the
reference algorithms (weights that sum to one, normalised Planck fractions, error paths).
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S


def _lw_const_sources(ngpt, nlay, ncol, B, tau):
    z = np.full((ngpt, nlay, ncol), B, np.float64)
    return {"lay_src": z, "lev_src_inc": z.copy(), "lev_src_dec": z.copy(),
            "sfc_src": np.full((ngpt, ncol), B)}, np.full((ngpt, nlay, ncol), tau)


@pytest.mark.parametrize("nmu", [1, 2, 3, 4])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_lw_transparent_atmosphere(oracle_mod, nmu, top_at_1):
    """tau = 0: no atmospheric emission; flux_up = pi * emis * B_sfc at every level."""
    O = oracle_mod
    ngpt, nlay, ncol = 4, 5, 3
    src, tau = _lw_const_sources(ngpt, nlay, ncol, 7.0, 0.0)
    emis = np.full((ncol, 2), 0.9)
    up, dn = O.rte_lw([[1, 2], [3, 4]], tau, top_at_1, src, emis, n_gauss_angles=nmu)
    np.testing.assert_allclose(dn, 0.0, atol=1e-12)
    np.testing.assert_allclose(up, np.pi * 0.9 * 7.0, rtol=1e-6)


@pytest.mark.parametrize("top_at_1", [True, False])
def test_lw_isothermal_black(oracle_mod, top_at_1):
    """Opaque isothermal atmosphere over a black surface: up = dn(surface) = pi B."""
    O = oracle_mod
    ngpt, nlay, ncol = 2, 6, 2
    src, tau = _lw_const_sources(ngpt, nlay, ncol, 3.0, 50.0)
    up, dn = O.rte_lw([[1, 2]], tau, top_at_1, src, np.ones((ncol, 1)))
    np.testing.assert_allclose(up, np.pi * 3.0, rtol=1e-10)
    sfc = nlay if top_at_1 else 0
    np.testing.assert_allclose(dn[:, sfc], np.pi * 3.0, rtol=1e-10)


def test_lw_incident_flux_passes_through(oracle_mod):
    O = oracle_mod
    src, tau = _lw_const_sources(1, 3, 2, 0.0, 0.0)
    inc = np.full((1, 2), 11.0)
    up, dn = O.rte_lw([[1, 1]], tau, True, src, np.ones((2, 1)), inc_flux=inc)
    np.testing.assert_allclose(dn, 11.0, rtol=1e-12)
    np.testing.assert_allclose(up, 0.0, atol=1e-12)


@pytest.mark.parametrize("top_at_1", [True, False])
def test_sw_no_scattering_direct_beam(oracle_mod, top_at_1):
    """ssa = 0, black surface: direct beam follows Beer's law, no diffuse radiation."""
    O = oracle_mod
    ngpt, nlay, ncol = 2, 4, 3
    tau = np.full((ngpt, nlay, ncol), 0.1)
    z = np.zeros_like(tau)
    mu0 = np.array([0.3, 0.6, 1.0])
    S0 = np.full((ngpt, ncol), 100.0)
    alb = np.zeros((ncol, 1))
    up, dn, dr = O.rte_sw([[1, 2]], tau, z, z, top_at_1, mu0, S0, alb, alb)
    depth = np.arange(nlay + 1) * 0.1
    if not top_at_1:
        depth = depth[::-1]
    expect = 100.0 * mu0[None, None, :] * np.exp(-depth[None, :, None] / mu0[None, None, :])
    np.testing.assert_allclose(dr, np.broadcast_to(expect, dr.shape), rtol=1e-12)
    np.testing.assert_allclose(dn, dr, atol=1e-12)
    np.testing.assert_allclose(up, 0.0, atol=1e-12)


def test_sw_conservative_white_surface(oracle_mod):
    """ssa = 1 and surface albedo 1: no absorption, so net flux vanishes at every level."""
    O = oracle_mod
    ngpt, nlay, ncol = 1, 8, 4
    rng = np.random.default_rng(0)
    tau = rng.uniform(0.01, 3.0, (ngpt, nlay, ncol))
    ssa = np.ones_like(tau)
    g = rng.uniform(0.0, 0.9, tau.shape)
    mu0 = rng.uniform(0.2, 1.0, ncol)
    S0 = np.full((ngpt, ncol), 500.0)
    alb = np.ones((ncol, 1))
    up, dn, dr = O.rte_sw([[1, 1]], tau, ssa, g, True, mu0, S0, alb, alb)
    net = dn - up
    assert np.max(np.abs(net)) < 1e-3 * 500.0


def test_planck_fractions_sum_to_band_planck(oracle_mod, tables):
    """Planck fractions are normalised per band and the fmajor weights sum to one, so the
    band sum of lay_src equals the band Planck function at T_lay (interpolate1D)."""
    O = oracle_mod
    lw = tables["lw"]
    kd = O.GasOptics(lw, S.ATM_GASES)
    atm = S.make_atmosphere(5, 12, seed=3, clouds=False)
    out = kd.gas_optics_lw(atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    tp = lw["totplnk"]
    tmin, tmax = lw["temp_ref"][0], lw["temp_ref"][-1]
    delta = (tmax - tmin) / (tp.shape[1] - 1)
    for b, (g0, g1) in enumerate(lw["bnd_limits_gpt"]):
        s = out["lay_src"][g0 - 1:g1].sum(axis=0)
        v0 = (atm["tlay"] - tmin) / delta
        frac = v0 - np.trunc(v0)
        idx = np.clip(np.trunc(v0).astype(int) + 1, 1, tp.shape[1] - 1)
        ref = tp[b, idx - 1] + frac * (tp[b, idx] - tp[b, idx - 1])
        np.testing.assert_allclose(s, ref, rtol=1e-12)


def test_gas_optics_physical_ranges(oracle_mod, tables):
    O = oracle_mod
    kd = O.GasOptics(tables["sw"], S.ATM_GASES)
    atm = S.make_atmosphere(6, 20, seed=4, clouds=False)
    out = kd.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    assert np.all(out["tau"] > 0)
    assert np.all((out["ssa"] >= 0) & (out["ssa"] <= 1))
    assert np.all(out["g"] == 0)
    np.testing.assert_allclose(out["toa_src"][:, 0], kd.solar_source())
    assert abs(kd.solar_source().sum() - 1360.8) < 5.0


def test_col_dry_matches_formula(oracle_mod):
    atm = S.make_atmosphere(4, 10, seed=5)
    h2o = atm["gases"]["h2o"]
    np.testing.assert_allclose(oracle_mod.get_col_dry(h2o, atm["plev"]), S.col_dry_from(h2o, atm["plev"]),
                               rtol=1e-14)


def test_missing_key_species_raises(oracle_mod, tables):
    with pytest.raises(oracle_mod.OracleError, match="required gas co2 is missing"):
        oracle_mod.GasOptics(tables["lw"], ["h2o", "o3", "n2o", "ch4", "o2", "n2"])


def test_gas_reduction(oracle_mod, tables):
    kd = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES)
    assert kd.ngas == len(S.ATM_GASES)
    # Intervals of absent minor gases (co, cfc11, cfc12) are dropped.
    lw = tables["lw"]
    drop = {"co", "cfc11", "cfc12"}
    keep_lo = sum(1 for g in lw["minor_gases_lower"] if g not in drop)
    assert kd.nminor_lower == keep_lo


def test_fluxes_byband_sum_to_broadband(oracle_mod):
    rng = np.random.default_rng(1)
    up = rng.uniform(0, 10, (8, 5, 3))
    dn = rng.uniform(0, 10, (8, 5, 3))
    bl = [[1, 3], [4, 4], [5, 8]]
    bb = oracle_mod.fluxes_broadband(up, dn)
    by = oracle_mod.fluxes_byband(bl, up, dn)
    np.testing.assert_allclose(by["bnd_flux_up"].sum(0), bb["flux_up"], rtol=1e-13)
    np.testing.assert_allclose(by["bnd_flux_net"].sum(0), bb["flux_net"], rtol=1e-12, atol=1e-12)
    # Each band includes its first g-point (the F90 behaviour).
    np.testing.assert_allclose(by["bnd_flux_dn"][1], dn[3], rtol=1e-15)


def test_heating_rate_sign_and_orientation(oracle_mod):
    plev = np.array([[100.0], [1000.0], [2000.0]])
    up = np.zeros((3, 1))
    dn = np.array([[10.0], [8.0], [8.0]])
    hr = oracle_mod.heating_rate(up, dn, plev)
    assert hr[0, 0] > 0 and hr[1, 0] == 0
    hr_flip = oracle_mod.heating_rate(up[::-1].copy(), dn[::-1].copy(), plev[::-1].copy())
    np.testing.assert_allclose(hr_flip[::-1], hr)


def test_cloud_optics_mask_and_combination(oracle_mod, tables):
    O = oracle_mod
    c = O.CloudOptics(tables["cloud_sw"])
    lwp = np.array([[0.0, 50.0, 0.0], [10.0, 0.0, 0.0]])
    iwp = np.array([[0.0, 0.0, 20.0], [5.0, 0.0, 0.0]])
    rel = np.full_like(lwp, 10.0)
    rei = np.full_like(lwp, 40.0)
    out = c.cloud_optics(lwp, iwp, rel, rei, two_stream=True)
    assert np.all(out["tau"][:, 0, 0] == 0)
    assert np.all(out["tau"][:, 0, 1] > 0) and np.all(out["tau"][:, 1, 0] > 0)
    one = c.cloud_optics(lwp, iwp, rel, rei, two_stream=False)
    np.testing.assert_allclose(one["tau"], out["tau"] * (1 - out["ssa"]), rtol=1e-10, atol=1e-14)


def test_forward_energy_budget(oracle_mod, tables):
    """Clear-sky column budgets of the synthetic configuration are physically sensible."""
    O = oracle_mod
    klw = O.GasOptics(tables["lw"], S.ATM_GASES)
    ksw = O.GasOptics(tables["sw"], S.ATM_GASES)
    atm = S.make_atmosphere(8, 30, seed=2, clouds=False)
    fl = O.forward_lw(klw, None, atm)
    fs = O.forward_sw(ksw, None, atm)
    assert 150 < fl["flux_up"][0].mean() < 350
    np.testing.assert_allclose(fs["flux_dn"][0], atm["mu0"] * ksw.solar_source().sum(), rtol=1e-12)
    assert np.all(fs["flux_up"][0] < fs["flux_dn"][0])


def test_solar_variability_formula(oracle_mod, tables):
    """set_solar_variability (src/Gas_optics_rrtmgp.cpp:745-760): quiet + (mg - 0.1495954)
    facular + (sb - 0.00066696) sunspot; the creation uses the table defaults, and the golden
    toa_src fixtures of the reference pin that default path."""
    t = tables["sw"]
    q, f, s = (np.asarray(t[k], np.float64) for k in ("solar_source_quiet", "solar_source_facular",
                                                      "solar_source_sunspot"))
    k = oracle_mod.GasOptics(t, S.ATM_GASES)
    want = q + (t["mg_default"] - 0.1495954) * f + (t["sb_default"] - 0.00066696) * s
    np.testing.assert_allclose(k.solar_source(), want, rtol=1e-15)
    for mg, sb in ((0.1495954, 0.00066696), (0.13, 400.0), (0.2, 2500.0)):
        k.set_solar_variability(mg, sb)
        np.testing.assert_allclose(k.solar_source(), q + (mg - 0.1495954) * f + (sb - 0.00066696) * s, rtol=1e-15)
    with pytest.raises(RuntimeError):
        oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).set_solar_variability(0.15, 900.0)
