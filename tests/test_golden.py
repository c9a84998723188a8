"""Pins the FP64 oracle to the reference implementation.

The fixtures in tests/golden were produced by the reference's own FP64 GPU classes
(rte-rrtmgp-cpp src_cuda/ + src_kernels_cuda/ built from its sources by oracle/ref/Makefile)
on the same seeded synthetic tables and inputs; tests/golden/make_ref_golden.py regenerates
them.  Tolerances: gas and cloud optics, add_to and flux sums agree to 1e-12 relative
(identical arithmetic up to operation order); the solvers to 1e-8 relative (CUDA and glibc
exp() differ by an ulp, amplified by eps/tau in the thin-layer source factor).
Known differences of the reference CUDA code that the oracle does not reproduce are asserted
explicitly (by-band sums skip each band's first g-point).
"""
from pathlib import Path

import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

GOLD = Path(__file__).resolve().parent / "golden"
sys_path_added = False

import importlib.util  # noqa: E402

_spec = importlib.util.spec_from_file_location("make_ref_golden", GOLD / "make_ref_golden.py")
G = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(G)
NCOL, NLAY = G.NCOL, G.NLAY


def load(name):
    p = GOLD / f"{name}.npz"
    if not p.exists():
        pytest.fail(f"missing golden fixture {p}")
    return np.load(p)


def relerr(a, b, floor_frac):
    floor = floor_frac * np.max(np.abs(b)) + 1e-300
    return float(np.max(np.abs(a - b) / (np.abs(b) + floor)))


@pytest.mark.parametrize("name,top,with_cd", [("gas_lw_top1", True, False), ("gas_lw_bot1", False, True)])
def test_gas_optics_lw_matches_reference(oracle_mod, tables, name, top, with_cd):
    ref = load(name)
    atm = S.make_atmosphere(NCOL, NLAY, seed=101, clouds=False, top_at_1=top)
    cd = S.col_dry_from(atm["gases"]["h2o"], atm["plev"]) if with_cd else None
    out = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"], cd)
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac"):
        assert relerr(out[k], ref[k], 1e-9) < 1e-12, k


@pytest.mark.parametrize("name,top", [("gas_sw_top1", True), ("gas_sw_bot1", False)])
def test_gas_optics_sw_matches_reference(oracle_mod, tables, name, top):
    ref = load(name)
    atm = S.make_atmosphere(NCOL, NLAY, seed=102, clouds=False, top_at_1=top)
    out = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES).gas_optics_sw(atm["play"], atm["plev"], atm["tlay"],
                                                                        atm["gases"])
    for k in ("tau", "ssa", "g", "toa_src"):
        assert relerr(out[k], ref[k], 1e-9) < 1e-12, k


@pytest.mark.parametrize("name,kind,two,delta", [("cloud_lw_1scl", "lw", False, False),
                                                 ("cloud_sw_2str", "sw", True, False),
                                                 ("cloud_sw_2str_delta", "sw", True, True)])
def test_cloud_optics_matches_reference(oracle_mod, tables, name, kind, two, delta):
    ref = load(name)
    atm = S.make_atmosphere(NCOL, NLAY, seed=103, clouds=True)
    out = oracle_mod.CloudOptics(tables["cloud_" + kind]).cloud_optics(atm["lwp"], atm["iwp"], atm["rel"],
                                                                       atm["rei"], two)
    if delta:
        oracle_mod.delta_scale(out["tau"], out["ssa"], out["g"])
    for k in out:
        assert relerr(out[k], ref[k], 1e-9) < 1e-12, k
    assert np.count_nonzero(ref["tau"]) > 0


def test_add_to_by_band_matches_reference(oracle_mod, tables):
    ref = load("add_to_2str_bybnd")
    gas, cld = G.addto_inputs()
    oracle_mod.add_to(tables["sw"]["bnd_limits_gpt"], gas, cld)
    for k in ("tau", "ssa", "g"):
        assert relerr(gas[k], ref[k], 1e-9) < 1e-12, k


def test_rte_lw_matches_reference(oracle_mod, tables):
    g = load("gas_lw_top1")
    ref = load("rte_lw_top1")
    up, dn = oracle_mod.rte_lw(tables["lw"]["bnd_limits_gpt"], g["tau"], True, {k: g[k] for k in g.files},
                               ref["emis"])
    assert relerr(up, ref["flux_up"], 1e-4) < 1e-8
    assert relerr(dn, ref["flux_dn"], 1e-4) < 1e-8


@pytest.mark.parametrize("name,gname,top", [("rte_sw_top1", "gas_sw_top1", True), ("rte_sw_bot1", "gas_sw_bot1", False)])
def test_rte_sw_matches_reference(oracle_mod, tables, name, gname, top):
    g = load(gname)
    ref = load(name)
    up, dn, dr = oracle_mod.rte_sw(tables["sw"]["bnd_limits_gpt"], g["tau"], g["ssa"], g["g"], top, ref["mu0"],
                                   g["toa_src"], ref["alb_dir"], ref["alb_dif"])
    assert relerr(dr, ref["flux_dir"], 1e-4) < 1e-8
    assert relerr(dn, ref["flux_dn"], 1e-4) < 1e-8
    assert relerr(up, ref["flux_up"], 1e-4) < 1e-8


def test_flux_reductions_match_reference(oracle_mod, tables):
    ref = load("fluxes")
    up, dn, dr = G.flux_inputs()
    bb = oracle_mod.fluxes_broadband(up, dn, dr)
    for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net"):
        assert relerr(bb[k], ref[k], 1e-9) < 1e-12, k
    # By band: the reference CUDA kernel sums g = band_lims(1,b) .. band_lims(2,b)-1 with the
    # 1-based limits used as 0-based indices, i.e. it skips each band's first g-point
    # (fluxes_kernels.cu:78-86).  The oracle follows the F90 (all g-points of the band); the
    # difference is exactly the first g-point of every band.
    bl = np.asarray(tables["sw"]["bnd_limits_gpt"])
    by = oracle_mod.fluxes_byband(bl, up, dn)
    first = bl[:, 0] - 1
    np.testing.assert_allclose(by["bnd_flux_up"] - up[first], ref["bnd_flux_up"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(by["bnd_flux_dn"] - dn[first], ref["bnd_flux_dn"], rtol=1e-12, atol=1e-12)


def test_aerosol_optics_matches_reference(oracle_mod):
    ref = load("aerosol_sw")
    atm = S.make_atmosphere(NCOL, NLAY, seed=107, clouds=False, top_at_1=False)
    aer, rh = G.aerosol_inputs(atm)
    out = oracle_mod.aerosol_optics(S.make_aerosol_luts(), aer, rh, atm["plev"])
    for k in ("tau", "ssa", "g"):
        assert relerr(out[k], ref[k], 1e-12) < 1e-13, k


# Dense minor-absorber layouts: the reference's gas optics on the dense tables (every
# halocarbon, up to 13 minor intervals in a band and 11 over one g-point), trace-gas
# atmospheres; make_ref_golden.py OUTDIR --only dense.
@pytest.mark.parametrize("name,kind,top,seed", [("gas_lw_dense_top1", "lw", True, 111),
                                                ("gas_lw_dense_bot1", "lw", False, 111),
                                                ("gas_sw_dense_top1", "sw", True, 112)])
def test_gas_optics_dense_matches_reference(oracle_mod, name, kind, top, seed):
    ref = load(name)
    atm = S.make_atmosphere(NCOL, NLAY, seed=seed, clouds=False, top_at_1=top, trace_gases=True)
    go = oracle_mod.GasOptics(S.make_kdist(kind, dense=True), S.ATM_GASES_DENSE)
    if kind == "lw":
        out = go.gas_optics_lw(atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
        keys = ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac")
    else:
        out = go.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
        keys = ("tau", "ssa", "g", "toa_src")
    for k in keys:
        assert relerr(out[k], ref[k], 1e-9) < 1e-12, k


def test_dense_tables_layout():
    """The dense tables carry what the fused kernels must accept: 13 intervals in one band,
    seven over the same g-points, intervals of every halocarbon."""
    for kind in ("lw", "sw"):
        d = S.make_kdist(kind, dense=True)
        lims = d["minor_limits_gpt_lower"]
        per_band = np.bincount((lims[:, 0] - 1) // 16, minlength=len(d["bnd_limits_gpt"]))
        assert per_band.max() >= 12
        cover = np.zeros(d["kmajor"].shape[-1], int)
        for a, b in lims:
            cover[a - 1:b] += 1
        assert cover.max() >= 6
        assert set(S.TRACE_GASES) <= set(d["gas_names"])
