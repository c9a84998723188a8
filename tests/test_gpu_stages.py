"""GPU parity of every per-stage C-ABI entry point against the FP64 oracle.

Each test runs the CUDA kernels through the C ABI (rrtmgp_b200.api -> librrtmgp_b200.so) and
the oracle on identical seeded inputs.  Tolerances (relative error |got - ref| / (|ref| + floor),
floor a fraction of max|ref|):
  optical properties / sources: FP64 1e-10 (summation order only), FP32 2e-4 (single
  precision interpolation weights), floor 1e-6;
  g-point fluxes: FP64 1e-8 -- the CUDA and glibc exp() differ by an ulp and the reference's
  (1 - T)/tau - T source factor amplifies that by eps/tau in thin layers -- and FP32 2e-4
  with a floor of 1% of the largest flux (an absolute W/m2 accuracy bound).
Shapes are ragged (ncol not a multiple of 32) on purpose.
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

pytestmark = pytest.mark.gpu

NCOL, NLAY = 37, 23
RTOL = {"f64": 1e-10, "f32": 2e-4}
FLUX_RTOL = {"f64": 1e-8, "f32": 2e-4}
FLUX_FLOOR = {"f64": 1e-4, "f32": 1e-2}


def T(x, dt, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dt, device=dev)


def N(t):
    return t.detach().double().cpu().numpy()


def dtypes():
    import torch
    return {"f32": torch.float32, "f64": torch.float64}


def cmp(name, got, ref, prec, floor_frac=1e-6, rtol=None):
    ref = np.asarray(ref, np.float64)
    got = np.asarray(got, np.float64)
    floor = max(floor_frac * np.max(np.abs(ref)), 1e-300)
    err = np.max(np.abs(got - ref) / (np.abs(ref) + floor))
    tol = RTOL[prec] if rtol is None else rtol
    assert err <= tol, f"{name}: max rel err {err:.3e} > {tol} ({prec}); max abs {np.max(np.abs(got - ref)):.3e}"


def cmp_flux(name, got, ref, prec):
    cmp(name, got, ref, prec, FLUX_FLOOR[prec], FLUX_RTOL[prec])


def gas_dict(atm, dt, dev, profile_o3=False):
    out = {}
    for k, v in atm["gases"].items():
        if v.size == 1:
            out[k] = T(v.reshape(1), dt, dev)
        elif profile_o3 and k == "o3":
            out[k] = T(v[:, 0].copy(), dt, dev)
        else:
            out[k] = T(v, dt, dev)
    return out


@pytest.fixture(scope="module")
def api(gpu):
    from rrtmgp_b200 import api
    return api


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("with_col_dry", [False, True])
def test_gas_optics_lw(api, oracle_mod, tables, gpu, prec, top_at_1, with_col_dry):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=11, clouds=False, top_at_1=top_at_1)
    cd = S.col_dry_from(atm["gases"]["h2o"], atm["plev"]) if with_col_dry else None
    ref = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"], cd)
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    got = kd.gas_optics_lw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                           T(atm["tsfc"], dt, gpu), gas_dict(atm, dt, gpu), T(atm["tlev"], dt, gpu),
                           None if cd is None else T(cd, dt, gpu))
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac"):
        cmp(k, N(got[k]), ref[k], prec)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_gas_optics_sw(api, oracle_mod, tables, gpu, prec, top_at_1):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=12, clouds=False, top_at_1=top_at_1)
    ref = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES).gas_optics_sw(
        atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    got = kd.gas_optics_sw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                           gas_dict(atm, dt, gpu, profile_o3=False))
    for k in ("tau", "ssa", "toa_src"):
        cmp(k, N(got[k]), ref[k], prec)
    assert float(got["g"].abs().max()) == 0.0


def _tables_with_band_crossing_minor(t):
    """Copy of an LW table set whose h2o_frgn interval [22, 30] (band 17-32, 1-based g) is
    moved to [28, 36], across the boundary with band 33-48: same contributor count, so the
    kminor columns stay valid.  Such a layout is outside the corner-packed tables."""
    t = dict(t)
    lims = np.array(t["minor_limits_gpt_lower"], copy=True)
    i = [n for n, (m, l) in enumerate(zip(t["minor_gases_lower"], lims))
         if m.strip() == "h2o_frgn" and tuple(l) == (22, 30)]
    assert i, "synthetic table layout changed"
    lims[i[0]] = (28, 36)
    t["minor_limits_gpt_lower"] = lims
    return t


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_gas_optics_lw_band_crossing_minor(api, oracle_mod, tables, gpu, prec):
    """A minor interval that spans two bands: the FP32 gas optics then runs the scalar-table
    kernel (the packed one needs intervals inside one band) and matches the oracle, and the
    fused forward, which needs the packed layout, refuses the table set."""
    import torch
    from rrtmgp_b200._abi import RrtmgpError, ERR_UNSUPPORTED
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    dt = dtypes()[prec]
    t = _tables_with_band_crossing_minor(tables["lw"])
    atm = S.make_atmosphere(NCOL, NLAY, seed=15, clouds=False)
    ref = oracle_mod.GasOptics(t, S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"], None)
    base_ref = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"], None)
    assert not np.allclose(ref["tau"], base_ref["tau"], rtol=1e-6)   # the move changes tau
    kd = api.Gas_optics_rrtmgp(t, S.ATM_GASES)
    got = kd.gas_optics_lw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                           T(atm["tsfc"], dt, gpu), gas_dict(atm, dt, gpu), T(atm["tlev"], dt, gpu), None)
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac"):
        cmp(k, N(got[k]), ref[k], prec)
    if prec == "f32":
        base = Radiation_solver(t, tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
        with pytest.raises(RrtmgpError) as e:
            Fused_solver(base).solve_lw(atm_to_device(atm, torch.float32, gpu), with_clouds=False)
        assert e.value.status == ERR_UNSUPPORTED


def test_gas_profile_and_scalar_inputs(api, oracle_mod, tables, gpu):
    """Gas_concs accepts scalars, (1, nlay) profiles and (ncol, nlay) fields."""
    import torch
    atm = S.make_atmosphere(NCOL, NLAY, seed=13, clouds=False)
    o3p = atm["gases"]["o3"][:, :1]
    atm["gases"]["o3"] = np.repeat(o3p, NCOL, axis=1)
    ref = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES).gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    g = gas_dict(atm, torch.float64, gpu, profile_o3=True)
    got = kd.gas_optics_sw(T(atm["play"], torch.float64, gpu), T(atm["plev"], torch.float64, gpu),
                           T(atm["tlay"], torch.float64, gpu), g)
    cmp("tau", N(got["tau"]), ref["tau"], "f64")


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_col_dry(api, gpu, prec):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=14)
    got = api.Gas_optics_rrtmgp.get_col_dry(T(atm["gases"]["h2o"], dt, gpu), T(atm["plev"], dt, gpu))
    cmp("col_dry", N(got), S.col_dry_from(atm["gases"]["h2o"], atm["plev"]), prec)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("kind", ["lw", "sw"])
def test_cloud_optics(api, oracle_mod, tables, gpu, prec, kind):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=15, clouds=True)
    two = kind == "sw"
    ref = oracle_mod.CloudOptics(tables["cloud_" + kind]).cloud_optics(atm["lwp"], atm["iwp"], atm["rel"], atm["rei"], two)
    c = api.Cloud_optics(tables["cloud_" + kind])
    got = c.cloud_optics(*(T(atm[k], dt, gpu) for k in ("lwp", "iwp", "rel", "rei")), two_stream=two)
    for k in ref:
        cmp(k, N(got[k]), ref[k], prec)


def _offset_tensor(x, dt, dev):
    """x on the device one element past a 16-byte boundary (a view into a larger buffer)."""
    import torch
    flat = torch.empty(x.size + 1, dtype=dt, device=dev)
    t = flat[1:].view(x.shape)
    t.copy_(torch.as_tensor(x, dtype=dt))
    return t


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("layout", ["ragged", "aligned", "offset"])
def test_delta_scale_and_add_to(api, oracle_mod, tables, gpu, prec, layout):
    """add_to takes 16-byte vector loads when ncol*nlay and the pointers allow ("aligned"),
    one value per thread otherwise (odd ncol*nlay: "ragged"; views off a 16-byte boundary)."""
    dt = dtypes()[prec]
    rng = np.random.default_rng(3)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    nb, ng = 14, 224
    nlay, ncol = (NLAY, NCOL) if layout == "ragged" else (24, 32)
    T_ = _offset_tensor if layout == "offset" else T
    gas = {"tau": rng.uniform(0, 2, (ng, nlay, ncol)), "ssa": rng.uniform(0, 1, (ng, nlay, ncol)),
           "g": rng.uniform(0, 0.9, (ng, nlay, ncol))}
    cld = {"tau": rng.uniform(0, 5, (nb, nlay, ncol)), "ssa": rng.uniform(0.5, 1, (nb, nlay, ncol)),
           "g": rng.uniform(0.7, 0.9, (nb, nlay, ncol))}
    cld["tau"][:, ::3] = 0.0
    ref_c = {k: v.copy() for k, v in cld.items()}
    oracle_mod.delta_scale(ref_c["tau"], ref_c["ssa"], ref_c["g"])
    got_c = {k: T_(v, dt, gpu) for k, v in cld.items()}
    api.delta_scale(got_c["tau"], got_c["ssa"], got_c["g"])
    for k in cld:
        cmp("delta_" + k, N(got_c[k]), ref_c[k], prec)
    ref_g = {k: v.copy() for k, v in gas.items()}
    oracle_mod.add_to(tables["sw"]["bnd_limits_gpt"], ref_g, ref_c)
    got_g = {k: T_(v, dt, gpu) for k, v in gas.items()}
    api.add_to(kd.bands, got_g, got_c)
    for k in gas:
        cmp("add_" + k, N(got_g[k]), ref_g[k], prec)
    # g-point by g-point, 1scl; and by band, 1scl
    ref1 = {"tau": gas["tau"].copy()}
    oracle_mod.add_to(None, ref1, {"tau": gas["tau"]})
    got1 = {"tau": T_(gas["tau"], dt, gpu)}
    api.add_to(kd.bands, got1, {"tau": T_(gas["tau"], dt, gpu)})
    cmp("add_1scl", N(got1["tau"]), ref1["tau"], prec)
    ref2 = {"tau": gas["tau"].copy()}
    oracle_mod.add_to(tables["sw"]["bnd_limits_gpt"], ref2, {"tau": cld["tau"]})
    got2 = {"tau": T_(gas["tau"], dt, gpu)}
    api.add_to(kd.bands, got2, {"tau": T_(cld["tau"], dt, gpu)})
    cmp("add_1scl_bybnd", N(got2["tau"]), ref2["tau"], prec)


def test_add_to_rejects_incompatible_shapes(api, tables, gpu):
    import torch
    from rrtmgp_b200._abi import RrtmgpError, ERR_ARG
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    a = {"tau": torch.zeros((224, 2, 3), dtype=torch.float64, device=gpu)}
    b = {"tau": torch.zeros((13, 2, 3), dtype=torch.float64, device=gpu)}
    with pytest.raises(RrtmgpError) as e:
        api.add_to(kd.bands, a, b)
    assert e.value.status == ERR_ARG and "incompatible band" in str(e.value)


def _lw_inputs(tables, oracle_mod, top_at_1, seed):
    atm = S.make_atmosphere(NCOL, NLAY, seed=seed, clouds=False, top_at_1=top_at_1)
    go = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    return atm, go


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("nmu", [1, 3])
@pytest.mark.parametrize("with_inc", [False, True])
def test_rte_lw(api, oracle_mod, tables, gpu, prec, top_at_1, nmu, with_inc):
    dt = dtypes()[prec]
    atm, go = _lw_inputs(tables, oracle_mod, top_at_1, 21)
    rng = np.random.default_rng(5)
    emis = rng.uniform(0.8, 1.0, (NCOL, 16))
    inc = rng.uniform(0, 2, (256, NCOL)) if with_inc else None
    bl = tables["lw"]["bnd_limits_gpt"]
    up, dn = oracle_mod.rte_lw(bl, go["tau"], top_at_1, go, emis, inc, nmu)
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    src = {k: T(v, dt, gpu) for k, v in go.items()}
    gu, gd = api.Rte_lw.rte_lw(kd.bands, src["tau"], top_at_1, src, T(emis, dt, gpu),
                               None if inc is None else T(inc, dt, gpu), nmu)
    cmp_flux("flux_up", N(gu), up, prec)
    cmp_flux("flux_dn", N(gd), dn, prec)


def test_rte_lw_large_nlay_without_smem_stash(api, oracle_mod, tables, gpu):
    """nlay large enough that the up-sweep stash does not fit in shared memory in FP64."""
    import torch
    dt = torch.float64
    ncol, nlay = 5, 400
    atm = S.make_atmosphere(ncol, nlay, seed=2, clouds=False)
    go = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    emis = np.full((ncol, 16), 0.95)
    up, dn = oracle_mod.rte_lw(tables["lw"]["bnd_limits_gpt"], go["tau"], True, go, emis)
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    src = {k: T(v, dt, gpu) for k, v in go.items()}
    gu, gd = api.Rte_lw.rte_lw(kd.bands, src["tau"], True, src, T(emis, dt, gpu))
    cmp_flux("flux_up", N(gu), up, "f64")
    cmp_flux("flux_dn", N(gd), dn, "f64")


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("nmu,nlay", [(1, NLAY), (3, NLAY), (1, 300)])
def test_rte_lw_surface_temperature_jacobian(api, oracle_mod, tables, gpu, prec, top_at_1, nmu, nlay):
    """gpt_flux_up_jac (the reference's do_jacobians output) against the oracle's, and against
    the finite difference it stands for: gpt_flux_up at Tsfc + 1 K minus at Tsfc (the fluxes
    depend on Tsfc only through the surface source, linearly).  One angle runs the chunked
    kernel up to 256 layers; three angles and 300 layers the per-(column, g-point) kernel."""
    import torch
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, nlay, seed=23, clouds=False, top_at_1=top_at_1)
    ko = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES)
    go = ko.gas_optics_lw(atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    emis = np.random.default_rng(6).uniform(0.8, 1.0, (NCOL, 16))
    bl = tables["lw"]["bnd_limits_gpt"]
    up, dn, jac = oracle_mod.rte_lw(bl, go["tau"], top_at_1, go, emis, None, nmu, flux_up_jac=True)
    go1 = ko.gas_optics_lw(atm["play"], atm["plev"], atm["tlay"], atm["tsfc"] + 1.0, atm["gases"], atm["tlev"])
    up1, _ = oracle_mod.rte_lw(bl, go1["tau"], top_at_1, go1, emis, None, nmu)
    np.testing.assert_allclose(jac, up1 - up, rtol=1e-9, atol=1e-9 * np.max(np.abs(jac)))
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    src = {k: T(v, dt, gpu) for k, v in go.items()}
    gu, gd, gj = api.Rte_lw.rte_lw(kd.bands, src["tau"], top_at_1, src, T(emis, dt, gpu), None, nmu,
                                   flux_up_jac=True)
    torch.cuda.synchronize()
    cmp_flux("flux_up", N(gu), up, prec)
    cmp_flux("flux_dn", N(gd), dn, prec)
    cmp_flux("flux_up_jac", N(gj), jac, prec)
    assert np.max(jac) > 0


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_solar_variability_matches_oracle(api, oracle_mod, tables, gpu, prec):
    """Gas_optics_rrtmgp_gpu::set_solar_variability (src_cuda/Gas_optics_rrtmgp.cu:1205-1217)
    at indices away from the table defaults: the solar source, get_tsi (its sum), toa_src of
    the gas optics and the fused shortwave forward against the oracle at the same indices,
    and a return to the defaults."""
    import torch
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=71, clouds=True)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    ko = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    g = gas_dict(atm, dt, gpu)
    for mg, sb in ((0.13, 400.0), (0.2, 2500.0), (tables["sw"]["mg_default"], tables["sw"]["sb_default"])):
        kd.set_solar_variability(mg, sb)
        ko.set_solar_variability(mg, sb)
        ref = ko.solar_source()
        assert abs(kd.get_tsi() - ref.sum()) <= 1e-12 * ref.sum()
        got = kd.gas_optics_sw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu), g)
        want = ko.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
        cmp("toa_src", N(got["toa_src"]), want["toa_src"], prec)
    if prec == "f32":
        from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
        base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
        base.ksw.set_solar_variability(0.2, 2500.0)
        ko.set_solar_variability(0.2, 2500.0)
        sw = Fused_solver(base).solve_sw(atm_to_device(atm, torch.float32, gpu))
        torch.cuda.synchronize()
        rsw = oracle_mod.forward_sw(ko, oracle_mod.CloudOptics(tables["cloud_sw"]), atm)
        for key in ("flux_up", "flux_dn", "flux_dn_dir"):
            e = float(np.max(np.abs(N(sw[key]) - rsw[key])))
            assert e < 5e-3, f"fused sw {key} at mg=0.2, sb=2500: {e:.3e} W/m2"


def _wait_timeouts():
    import ctypes
    from rrtmgp_b200 import _abi
    n = ctypes.c_uint(0)
    assert _abi.load().rrtmgp_b200_device_wait_timeouts(ctypes.byref(n)) == 0
    return n.value


@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("ncol,nlay", [(36, 23), (68, 128), (4, 129), (100, 192), (2048, 40)])
@pytest.mark.parametrize("with_inc", [False, True])
def test_rte_lw_tma_tiles(api, oracle_mod, tables, gpu, top_at_1, ncol, nlay, with_inc):
    """FP32, one angle, ncol a multiple of 4 and nlay <= 192: the solver copies its layer inputs
    with TMA tiles of 32 columns x nlay layers (column tiles with idle lanes, 8- and 16-layer
    chunks, several tiles per persistent block so both copy stages cycle).  Fluxes and the
    surface-temperature Jacobian against the oracle, and bit-identical to the kernel that reads
    global memory directly, which runs on ncol + 1 columns (not a multiple of 4) of the same
    atmosphere; no copy timed out."""
    import torch
    dt = torch.float32
    before = _wait_timeouts()
    n1 = ncol + 1
    atm = S.make_atmosphere(n1, nlay, seed=40 + nlay, clouds=False, top_at_1=top_at_1)
    go = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    rng = np.random.default_rng(nlay)
    emis = rng.uniform(0.8, 1.0, (n1, 16))
    inc = rng.uniform(0, 2, (256, n1)) if with_inc else None
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    keys = ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac")
    full = {k: T(go[k], dt, gpu) for k in keys}
    part = {k: T(go[k][..., :ncol], dt, gpu) for k in keys}
    ref = api.Rte_lw.rte_lw(kd.bands, full["tau"], top_at_1, full, T(emis, dt, gpu),
                            None if inc is None else T(inc, dt, gpu), 1, flux_up_jac=True)
    got = api.Rte_lw.rte_lw(kd.bands, part["tau"], top_at_1, part, T(emis[:ncol], dt, gpu),
                            None if inc is None else T(inc[:, :ncol], dt, gpu), 1, flux_up_jac=True)
    torch.cuda.synchronize()
    for name, g, r in zip(("flux_up", "flux_dn", "flux_up_jac"), got, ref):
        assert torch.equal(g, r[..., :ncol]), f"{name}: TMA and direct kernels differ"
    sub = {k: v[..., :ncol] for k, v in go.items()}
    up, dn, jac = oracle_mod.rte_lw(tables["lw"]["bnd_limits_gpt"], sub["tau"], top_at_1, sub, emis[:ncol],
                                    None if inc is None else inc[:, :ncol], 1, flux_up_jac=True)
    cmp_flux("flux_up", N(got[0]), up, "f32")
    cmp_flux("flux_dn", N(got[1]), dn, "f32")
    cmp_flux("flux_up_jac", N(got[2]), jac, "f32")
    assert _wait_timeouts() == before


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("with_dif", [False, True])
def test_rte_sw(api, oracle_mod, tables, gpu, prec, top_at_1, with_dif):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(NCOL, NLAY, seed=31, clouds=True, top_at_1=top_at_1)
    ko = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    go = ko.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    c = oracle_mod.CloudOptics(tables["cloud_sw"]).cloud_optics(atm["lwp"], atm["iwp"], atm["rel"], atm["rei"], True)
    oracle_mod.delta_scale(c["tau"], c["ssa"], c["g"])
    bl = tables["sw"]["bnd_limits_gpt"]
    oracle_mod.add_to(bl, go, c)
    rng = np.random.default_rng(9)
    alb_dir = rng.uniform(0.05, 0.3, (NCOL, 14))
    alb_dif = rng.uniform(0.05, 0.3, (NCOL, 14))
    inc_dif = rng.uniform(0, 1, (224, NCOL)) if with_dif else None
    up, dn, dr = oracle_mod.rte_sw(bl, go["tau"], go["ssa"], go["g"], top_at_1, atm["mu0"], go["toa_src"],
                                   alb_dir, alb_dif, inc_dif)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    gu, gd, gr = api.Rte_sw.rte_sw(kd.bands, T(go["tau"], dt, gpu), T(go["ssa"], dt, gpu), T(go["g"], dt, gpu),
                                   top_at_1, T(atm["mu0"], dt, gpu), T(go["toa_src"], dt, gpu),
                                   T(alb_dir, dt, gpu), T(alb_dif, dt, gpu),
                                   None if inc_dif is None else T(inc_dif, dt, gpu))
    cmp_flux("flux_dir", N(gr), dr, prec)
    cmp_flux("flux_dn", N(gd), dn, prec)
    cmp_flux("flux_up", N(gu), up, prec)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("nlay", [129, 200, 257])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_rte_deep_columns(api, oracle_mod, tables, gpu, prec, nlay, top_at_1):
    """Layer counts around the solvers' kernel switches: the chunked kernels take 16-layer
    chunks above 128 layers (the FP64 shortwave switches to one thread per column and g-point
    there) and both solvers switch to one thread per column and g-point above 256."""
    _gas_optics_and_rte(api, oracle_mod, tables, gpu, prec, 33, nlay, top_at_1)


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("ncol,nlay", [(1, 2), (2, 3), (1, 9)])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_rte_small_domains(api, oracle_mod, tables, gpu, prec, ncol, nlay, top_at_1):
    """Domains of one or two columns and a few layers: gas optics and both solvers with most
    lanes of every warp and most layers of every chunk idle."""
    _gas_optics_and_rte(api, oracle_mod, tables, gpu, prec, ncol, nlay, top_at_1)


def _gas_optics_and_rte(api, oracle_mod, tables, gpu, prec, ncol, nlay, top_at_1):
    dt = dtypes()[prec]
    atm = S.make_atmosphere(ncol, nlay, seed=nlay, clouds=True, top_at_1=top_at_1)
    kd_lw = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    go = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    g_lw = kd_lw.gas_optics_lw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                               T(atm["tsfc"], dt, gpu), gas_dict(atm, dt, gpu), T(atm["tlev"], dt, gpu), None)
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac"):
        cmp("gas lw " + k, N(g_lw[k]), go[k], prec)
    emis = np.random.default_rng(nlay).uniform(0.8, 1.0, (ncol, 16))
    up, dn = oracle_mod.rte_lw(tables["lw"]["bnd_limits_gpt"], go["tau"], top_at_1, go, emis)
    src = {k: T(v, dt, gpu) for k, v in go.items()}
    gu, gd = api.Rte_lw.rte_lw(kd_lw.bands, src["tau"], top_at_1, src, T(emis, dt, gpu))
    cmp_flux("lw flux_up", N(gu), up, prec)
    cmp_flux("lw flux_dn", N(gd), dn, prec)

    ko = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    gs = ko.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    kd_sw = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    g_sw = kd_sw.gas_optics_sw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                               gas_dict(atm, dt, gpu))
    for k in ("tau", "ssa", "toa_src"):
        cmp("gas sw " + k, N(g_sw[k]), gs[k], prec)
    c = oracle_mod.CloudOptics(tables["cloud_sw"]).cloud_optics(atm["lwp"], atm["iwp"], atm["rel"], atm["rei"], True)
    oracle_mod.delta_scale(c["tau"], c["ssa"], c["g"])
    bl = tables["sw"]["bnd_limits_gpt"]
    oracle_mod.add_to(bl, gs, c)
    rng = np.random.default_rng(nlay + 1)
    alb_dir = rng.uniform(0.05, 0.3, (ncol, 14))
    alb_dif = rng.uniform(0.05, 0.3, (ncol, 14))
    inc_dif = rng.uniform(0, 1, (224, ncol))
    up, dn, dr = oracle_mod.rte_sw(bl, gs["tau"], gs["ssa"], gs["g"], top_at_1, atm["mu0"], gs["toa_src"],
                                   alb_dir, alb_dif, inc_dif)
    gu, gd, gr = api.Rte_sw.rte_sw(kd_sw.bands, T(gs["tau"], dt, gpu), T(gs["ssa"], dt, gpu), T(gs["g"], dt, gpu),
                                   top_at_1, T(atm["mu0"], dt, gpu), T(gs["toa_src"], dt, gpu),
                                   T(alb_dir, dt, gpu), T(alb_dif, dt, gpu), T(inc_dif, dt, gpu))
    cmp_flux("sw flux_dir", N(gr), dr, prec)
    cmp_flux("sw flux_dn", N(gd), dn, prec)
    cmp_flux("sw flux_up", N(gu), up, prec)


def test_rte_sw_workspace_required(api, tables, gpu):
    """Columns deeper than the on-chip solver's limit (256 layers in FP32) need the caller's
    workspace and are refused without one; shallower columns need none."""
    import torch
    from rrtmgp_b200._abi import RrtmgpError, ERR_WORKSPACE
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    m = torch.ones(2, dtype=torch.float32, device=gpu)
    a = torch.zeros((2, 14), dtype=torch.float32, device=gpu)
    s = torch.ones((224, 2), dtype=torch.float32, device=gpu)
    small = torch.empty(16, dtype=torch.uint8, device=gpu)
    deep = torch.zeros((224, 257, 2), dtype=torch.float32, device=gpu)
    with pytest.raises(RrtmgpError) as e:
        api.Rte_sw.rte_sw(kd.bands, deep, deep, deep, True, m, s, a, a, workspace=small)
    assert e.value.status == ERR_WORKSPACE
    none = torch.empty(0, dtype=torch.uint8, device=gpu)
    z = torch.zeros((224, 3, 2), dtype=torch.float32, device=gpu)
    up, dn, dr = api.Rte_sw.rte_sw(kd.bands, z, z, z, True, m, s, a, a, workspace=none)
    torch.cuda.synchronize()
    assert torch.allclose(dr[:, -1, :], s)   # tau = 0: the direct beam reaches the surface unchanged


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_fluxes_and_heating_rate(api, oracle_mod, tables, gpu, prec):
    dt = dtypes()[prec]
    rng = np.random.default_rng(4)
    up = rng.uniform(0, 20, (224, NLAY + 1, NCOL))
    dn = rng.uniform(0, 20, (224, NLAY + 1, NCOL))
    dr = rng.uniform(0, 20, (224, NLAY + 1, NCOL))
    ref = oracle_mod.fluxes_broadband(up, dn, dr)
    got = api.Fluxes_broadband.reduce(T(up, dt, gpu), T(dn, dt, gpu), T(dr, dt, gpu))
    for k in ref:
        cmp(k, N(got[k]), ref[k], prec, floor_frac=1e-3)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    bl = tables["sw"]["bnd_limits_gpt"]
    refb = oracle_mod.fluxes_byband(bl, up, dn, dr)
    gotb = api.Fluxes_byband.reduce(kd.bands, T(up, dt, gpu), T(dn, dt, gpu), T(dr, dt, gpu))
    for k in refb:
        cmp(k, N(gotb[k]), refb[k], prec, floor_frac=1e-3)
    atm = S.make_atmosphere(NCOL, NLAY, seed=3)
    hr = api.heating_rate(got["flux_up"], got["flux_dn"], T(atm["plev"], dt, gpu))
    href = oracle_mod.heating_rate(N(got["flux_up"]), N(got["flux_dn"]), atm["plev"])
    cmp("heating_rate", N(hr), href, "f64" if prec == "f64" else "f32", floor_frac=1e-3)


def test_range_check(api, tables, gpu):
    import torch
    from rrtmgp_b200._abi import RrtmgpError, ERR_RANGE
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    atm = S.make_atmosphere(8, 6, seed=1)
    args = [T(atm[k], torch.float64, gpu) for k in ("play", "plev", "tlay", "tlev")]
    kd.check_range(args[0], args[1], args[2], args[3], T(atm["tsfc"], torch.float64, gpu))
    bad = atm["tlay"].copy()
    bad[2, 3] = 400.0
    with pytest.raises(RrtmgpError) as e:
        kd.check_range(args[0], args[1], T(bad, torch.float64, gpu), args[3])
    assert e.value.status == ERR_RANGE and "tlay is out of range" in str(e.value)


def test_missing_gas_is_reported(api, tables, gpu):
    import torch
    from rrtmgp_b200._abi import RrtmgpError, ERR_MISSING_GAS
    with pytest.raises(RrtmgpError) as e:
        api.Gas_optics_rrtmgp(tables["lw"], ["h2o", "o3"])
    assert e.value.status == ERR_MISSING_GAS and "required gas co2 is missing" in str(e.value)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    atm = S.make_atmosphere(4, 5, seed=1)
    g = gas_dict(atm, torch.float64, gpu)
    del g["ch4"]
    with pytest.raises(RrtmgpError) as e:
        kd.gas_optics_sw(T(atm["play"], torch.float64, gpu), T(atm["plev"], torch.float64, gpu),
                         T(atm["tlay"], torch.float64, gpu), g)
    assert e.value.status == ERR_MISSING_GAS


@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("ncol,nlay", [(37, 23), (300, 128), (5, 2)])
def test_rte_sw_absorbed_flux_heating_rate(api, tables, gpu, top_at_1, ncol, nlay):
    """rte_sw_abs returns rte_sw's fluxes plus each layer's absorbed flux per g-point, and the
    heating rate summed from it equals heating_rate_sw_layers' (which recomputes the two-stream
    from tau, ssa and g).  FP32: the fluxes within 2e-5 relative (the two kernel instances round
    differently in the last bits), the heating rates within 2e-3 K/day + 1e-4 relative.  Deeper
    than 128 layers is refused with RRTMGP_B200_ERR_UNSUPPORTED before any launch."""
    import torch
    from rrtmgp_b200 import _abi
    dt = torch.float32
    lib = _abi.load()
    P, st = api._ptr, api._stream()
    atm = S.make_atmosphere(ncol, nlay, seed=41, clouds=False, top_at_1=top_at_1)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    go = kd.gas_optics_sw(T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu),
                          gas_dict(atm, dt, gpu))
    mu0, plev = T(atm["mu0"], dt, gpu), T(atm["plev"], dt, gpu)
    alb_dir, alb_dif = T(atm["sfc_alb_dir"], dt, gpu), T(atm["sfc_alb_dif"], dt, gpu)
    up, dn, dr = api.Rte_sw.rte_sw(kd.bands, go["tau"], go["ssa"], go["g"], top_at_1, mu0, go["toa_src"],
                                   alb_dir, alb_dif)
    ng = go["tau"].shape[0]
    hr_ref = torch.empty((nlay, ncol), dtype=dt, device=gpu)
    _abi.check(lib.rrtmgp_b200_heating_rate_sw_layers_f32(
        ncol, nlay, ng, int(top_at_1), P(go["tau"]), P(go["ssa"]), P(go["g"]), P(mu0), P(up), P(dn), P(dr),
        P(plev), P(hr_ref), st))
    up2, dn2, dr2 = (torch.empty_like(up) for _ in range(3))
    layer_abs = torch.empty_like(go["tau"])
    hr = torch.empty((nlay, ncol), dtype=dt, device=gpu)
    _abi.check(lib.rrtmgp_b200_rte_sw_abs_f32(
        kd.bands.handle, ncol, nlay, int(top_at_1), P(go["tau"]), P(go["ssa"]), P(go["g"]), P(mu0),
        P(go["toa_src"]), P(alb_dir), P(alb_dif), None, P(up2), P(dn2), P(dr2), P(layer_abs), st))
    _abi.check(lib.rrtmgp_b200_heating_rate_from_layer_abs_f32(ncol, nlay, ng, P(layer_abs), P(plev), P(hr), st))
    torch.cuda.synchronize()
    for name, a, b in (("flux_up", up2, up), ("flux_dn", dn2, dn), ("flux_dir", dr2, dr)):
        cmp(name, N(a), N(b), "f32", floor_frac=1e-6, rtol=2e-5)
    err = np.abs(N(hr) - N(hr_ref))
    bound = 2e-3 + 1e-4 * np.abs(N(hr_ref))
    assert np.all(err <= bound), f"heating rate: max diff {err.max():.3e} K/day"
    if nlay == 128:
        t = T(np.zeros((ng, 129, ncol)), dt, gpu)
        f = T(np.zeros((ng, 130, ncol)), dt, gpu)
        status = lib.rrtmgp_b200_rte_sw_abs_f32(
            kd.bands.handle, ncol, 129, int(top_at_1), P(t), P(t), P(t), P(mu0), P(go["toa_src"]), P(alb_dir),
            P(alb_dif), None, P(f), P(f), P(f), P(t), st)
        assert status == _abi.ERR_UNSUPPORTED and b"128 layers" in lib.rrtmgp_b200_last_error()
