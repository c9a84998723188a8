"""Seeded synthetic RRTMGP-style coefficient tables and atmospheres.

The real k-distribution files (``rrtmgp-gas-lw-g256.nc``, ``rrtmgp-gas-sw-g224.nc``) and
cloud look-up tables are not available, so this module builds stand-ins with the same
netCDF schema that ``load_and_init_gas_optics`` / ``load_and_init_cloud_optics`` read in
the reference (src_test/Radiation_solver.cpp:70-329).  Every array is returned in the
*file* layout (C order, numpy shape = netCDF dimension order), i.e. exactly the memory the
reference's ``Array<Float,N>`` holds after ``get_variable`` (Fortran order, first dim
fastest), so real tables can be dropped in unchanged.

  kmajor            (temperature, pressure_interp, mixing_fraction, gpt)     -> g fastest
  plank_fraction    (temperature, pressure_interp, mixing_fraction, gpt)
  kminor_lower      (temperature, mixing_fraction, contributors_lower)
  rayl_lower/upper  (temperature, mixing_fraction, gpt)
  vmr_ref           (temperature, absorber_ext, atmos_layer)
  key_species       (bnd, atmos_layer, pair)
  bnd_limits_gpt    (bnd, pair)          1-based inclusive
  minor_limits_gpt_lower (minor_absorber_intervals_lower, pair)
  totplnk           (bnd, temperature_Planck)
  lut_extliq        (nband, nsize_liq);  lut_extice (nrghice, nband, nsize_ice)

Dimensions follow the public g256/g224 files: 16 LW bands x 16 g-points, 14 SW bands x
16 g-points, 14 reference temperatures (160..355 K), 59 reference pressures
(109663 Pa .. 1.005 Pa, log spaced), 9 mixing fractions, 196 Planck temperatures.
"""
from __future__ import annotations

import numpy as np

GAS_NAMES = ["h2o", "co2", "o3", "n2o", "co", "ch4", "o2", "n2", "cfc11", "cfc12"]
# Gases present in the synthetic atmospheres (co, cfc11, cfc12 are absent on purpose so the
# k-distribution constructor's gas/minor-absorber reduction is exercised).
ATM_GASES = ["h2o", "co2", "o3", "n2o", "ch4", "o2", "n2"]
# The dense tables (make_kdist(..., dense=True)) list every gas of the public LW g256 file,
# halocarbons included, and the trace-gas atmospheres (make_atmosphere(..., trace_gases=True))
# carry all of them.
TRACE_GASES = ["ccl4", "cfc22", "hfc143a", "hfc125", "hfc23", "hfc32", "hfc134a", "cf4", "no2"]
GAS_NAMES_DENSE = GAS_NAMES + TRACE_GASES
ATM_GASES_DENSE = ATM_GASES + ["co", "cfc11", "cfc12"] + TRACE_GASES
_TRACE_VMR = {"co": 1.2e-7, "cfc11": 2.3e-10, "cfc12": 5.2e-10, "ccl4": 8.0e-11, "cfc22": 2.5e-10,
              "hfc143a": 2.0e-11, "hfc125": 2.5e-11, "hfc23": 3.0e-11, "hfc32": 1.5e-11,
              "hfc134a": 1.0e-10, "cf4": 8.0e-11, "no2": 1.0e-9}

LW_BAND_WVN = [(10, 250), (250, 500), (500, 630), (630, 700), (700, 820), (820, 980),
               (980, 1080), (1080, 1180), (1180, 1390), (1390, 1480), (1480, 1800),
               (1800, 2080), (2080, 2250), (2250, 2390), (2390, 2680), (2680, 3250)]
SW_BAND_WVN = [(820, 2680), (2680, 3250), (3250, 4000), (4000, 4650), (4650, 5150),
               (5150, 6150), (6150, 7700), (7700, 8050), (8050, 12850), (12850, 16000),
               (16000, 22650), (22650, 29000), (29000, 38000), (38000, 50000)]

NTEMP = 14
NPRES = 59
NETA = 9
NPLANCK = 196
PRESS_REF_MAX = 109663.3
PRESS_REF_MIN = 1.005183574463
PRESS_REF_TROP = 9948.431564193395
# Top-of-atmosphere level pressure used by the synthetic atmospheres: the 1 Pa top asked for
# by the benchmark configs lies below the table minimum, which the reference range check
# rejects (src/Gas_optics_rrtmgp.cpp:815-816), so it is clamped just above press_ref_min.
P_TOP = 1.0052

# 1-based indices into GAS_NAMES; 0 = no species.  (lower pair, upper pair) per band.
_LW_KEY = [((1, 2), (1, 2)), ((1, 2), (1, 2)), ((1, 2), (4, 2)), ((1, 2), (1, 2)),
           ((1, 3), (3, 2)), ((1, 2), (3, 2)), ((1, 3), (3, 2)), ((1, 3), (3, 2)),
           ((1, 4), (6, 2)), ((1, 6), (6, 2)), ((1, 0), (0, 0)), ((1, 2), (3, 2)),
           ((1, 2), (3, 2)), ((4, 2), (4, 2)), ((1, 2), (4, 2)), ((1, 6), (6, 2))]
_SW_KEY = [((1, 2), (1, 2)), ((1, 6), (1, 6)), ((1, 2), (1, 2)), ((1, 2), (1, 2)),
           ((1, 6), (1, 6)), ((1, 2), (1, 2)), ((1, 7), (1, 7)), ((1, 2), (1, 2)),
           ((1, 7), (1, 7)), ((1, 7), (3, 7)), ((1, 7), (3, 7)), ((1, 3), (3, 7)),
           ((3, 7), (3, 7)), ((3, 7), (3, 0))]

_MINOR_IDS = ["h2o_frgn", "h2o_self", "co2", "o3", "n2o", "co", "ch4", "o2", "n2", "cfc11",
              "cfc12", "o2_n2"]
_MINOR_GAS = ["h2o", "h2o", "co2", "o3", "n2o", "co", "ch4", "o2", "n2", "cfc11", "cfc12",
              "o2"]
_MINOR_IDS_DENSE = _MINOR_IDS + ["co2_n2", "n2_o2"] + TRACE_GASES
_MINOR_GAS_DENSE = _MINOR_GAS + ["co2", "n2"] + TRACE_GASES

_H = 6.62607015e-34
_C = 2.99792458e8
_KB = 1.380649e-23


def _planck_band_radiance(wvn_lo, wvn_hi, temps, nsub=400):
    """Band-integrated Planck radiance [W m-2 sr-1] between two wavenumbers [cm-1]."""
    nu = np.linspace(wvn_lo, wvn_hi, nsub + 1) * 100.0  # m-1
    nu_mid = 0.5 * (nu[1:] + nu[:-1])
    dnu = np.diff(nu)
    t = np.asarray(temps, dtype=np.float64)[:, None]
    x = _H * _C * nu_mid[None, :] / (_KB * t)
    b = 2.0 * _H * _C ** 2 * nu_mid[None, :] ** 3 / np.expm1(x)
    return (b * dnu[None, :]).sum(axis=1)


def _ref_grids():
    press_ref = np.exp(np.linspace(np.log(PRESS_REF_MAX), np.log(PRESS_REF_MIN), NPRES))
    press_ref[-1] = PRESS_REF_MIN
    temp_ref = 160.0 + 15.0 * np.arange(NTEMP)
    return press_ref, temp_ref


def _minor_intervals(rng, band_lims, atm):
    """Minor-absorber intervals inside bands: list of dicts (file order)."""
    out = []
    for ib, (g0, g1) in enumerate(band_lims):
        nint = rng.integers(1, 4)
        for _ in range(nint):
            mid = rng.integers(0, len(_MINOR_IDS))
            ident = _MINOR_IDS[mid]
            ng = int(rng.integers(4, g1 - g0 + 2))
            start = int(rng.integers(g0, g1 - ng + 2))
            if ident in ("h2o_frgn", "h2o_self"):
                dens, sgas, comp = 1, "h2o", 1 if ident == "h2o_frgn" else 0
            elif ident == "o2_n2":
                dens, sgas, comp = 1, "n2", 0
            else:
                dens = int(rng.integers(0, 2))
                sgas = "" if (atm == 1 or rng.random() < 0.5) else "h2o"
                comp = int(rng.integers(0, 2)) if sgas else 0
            out.append(dict(id=ident, lims=(start, start + ng - 1), dens=dens, sgas=sgas,
                            comp=comp))
    return out


def _minor_intervals_dense(rng, band_lims, atm):
    """Minor-absorber intervals of the dense tables: 2-5 per band, 13 in band 0, and in bands 3
    and 9 seven intervals that all cover the whole band (seven on the same g-points), drawn
    over every minor absorber including the halocarbons, as the public LW g256 file lists many
    absorbers over the same g-points."""
    out = []
    for ib, (g0, g1) in enumerate(band_lims):
        nint = 13 if ib == 0 else (7 if ib in (3, 9) else int(rng.integers(2, 6)))
        for _ in range(nint):
            mid = int(rng.integers(0, len(_MINOR_IDS_DENSE)))
            ident = _MINOR_IDS_DENSE[mid]
            if ib in (3, 9):
                start, ng = g0, g1 - g0 + 1
            else:
                ng = int(rng.integers(2, g1 - g0 + 2))
                start = int(rng.integers(g0, g1 - ng + 2))
            if ident in ("h2o_frgn", "h2o_self"):
                dens, sgas, comp = 1, "h2o", 1 if ident == "h2o_frgn" else 0
            elif ident in ("o2_n2", "co2_n2"):
                dens, sgas, comp = 1, "n2", 0
            elif ident == "n2_o2":
                dens, sgas, comp = 1, "o2", 0
            else:
                dens = int(rng.integers(0, 2))
                sgas = "" if (atm == 1 or rng.random() < 0.5) else "h2o"
                comp = int(rng.integers(0, 2)) if sgas else 0
            out.append(dict(id=ident, lims=(start, start + ng - 1), dens=dens, sgas=sgas, comp=comp))
    return out


def make_kdist(kind: str, seed: int = 1, dense: bool = False):
    """Return a dict with the reference netCDF variables for an LW or SW k-distribution.

    dense=True: the gas list of the public LW g256 file (halocarbons included) and a dense
    minor-absorber layout (_minor_intervals_dense); the default tables keep 1-3 intervals per
    band."""
    assert kind in ("lw", "sw")
    rng = np.random.default_rng(seed + (0 if kind == "lw" else 1000))
    gas_names = GAS_NAMES_DENSE if dense else GAS_NAMES
    wvn = LW_BAND_WVN if kind == "lw" else SW_BAND_WVN
    keys = _LW_KEY if kind == "lw" else _SW_KEY
    nband = len(wvn)
    ngpb = 16
    ngpt = nband * ngpb
    band_lims_gpt = np.array([[1 + b * ngpb, (b + 1) * ngpb] for b in range(nband)], np.int32)
    press_ref, temp_ref = _ref_grids()
    ngas = len(gas_names)

    key_species = np.zeros((nband, 2, 2), np.int32)
    for b, (lo, up) in enumerate(keys):
        key_species[b, 0, :] = lo
        key_species[b, 1, :] = up

    # vmr_ref (ntemp, ngas+1, 2): reference volume mixing ratios; index 0 is dry air.
    base_vmr = {"h2o": 3e-3, "co2": 4e-4, "o3": 5e-7, "n2o": 3e-7, "co": 1e-7, "ch4": 1.8e-6,
                "o2": 0.2095, "n2": 0.7808, "cfc11": 2e-10, "cfc12": 5e-10}
    base_vmr.update({g: _TRACE_VMR[g] for g in TRACE_GASES})
    vmr_ref = np.zeros((NTEMP, ngas + 1, 2))
    vmr_ref[:, 0, :] = 1.0
    for i, gname in enumerate(gas_names):
        for atm in range(2):
            fac = (1.0 if atm == 0 else (0.002 if gname == "h2o" else (8.0 if gname == "o3" else 1.0)))
            vmr_ref[:, i + 1, atm] = base_vmr[gname] * fac * (1.0 + 0.02 * np.linspace(-1, 1, NTEMP))

    # kmajor (ntemp, npres+1, neta, ngpt): per-molecule absorption [cm2], smooth in T, p, eta,
    # increasing across the g-points of a band (k-distribution ordering).
    tt = ((temp_ref - 250.0) / 100.0)[:, None, None, None]
    pgrid = np.concatenate([press_ref, [press_ref[-1]]])
    pp = np.log10(pgrid / 1e4)[None, :, None, None]
    ee = np.linspace(0.0, 1.0, NETA)[None, None, :, None]
    gfrac = np.tile(np.linspace(0.0, 1.0, ngpb), nband)[None, None, None, :]
    if kind == "lw":
        band_base = np.array([-20.6, -20.9, -21.3, -20.8, -21.9, -23.6, -23.2, -23.4, -21.6,
                              -21.2, -20.7, -21.8, -22.4, -20.9, -22.6, -21.9])
    else:
        band_base = np.array([-21.2, -21.6, -22.6, -22.3, -21.9, -22.1, -22.9, -23.3, -23.6,
                              -24.2, -24.9, -24.6, -22.9, -21.7])
    band_base = band_base - (2.4 if kind == "lw" else 4.0)
    bb = np.repeat(band_base, ngpb)[None, None, None, :]
    gslope = np.repeat(rng.uniform(2.6, 3.8, nband) if kind == "lw" else rng.uniform(2.0, 3.2, nband),
                       ngpb)[None, None, None, :]
    palpha = np.repeat(rng.uniform(0.1, 0.8, nband), ngpb)[None, None, None, :]
    wig = 0.15 * np.sin(2.0 * np.pi * (ee * 1.3 + gfrac * 0.7 + tt * 0.4))
    log10k = bb + gslope * gfrac ** 2 + 0.35 * tt + palpha * gfrac * pp + 0.6 * (ee - 0.5) + wig
    kmajor = 10.0 ** log10k
    kmajor = np.ascontiguousarray(kmajor)

    # Minor absorbers.
    def minor_block(atm):
        ints = (_minor_intervals_dense if dense else _minor_intervals)(rng, band_lims_gpt.tolist(), atm)
        ncontrib = sum(iv["lims"][1] - iv["lims"][0] + 1 for iv in ints)
        kmin = np.empty((NTEMP, NETA, ncontrib))
        start = []
        off = 0
        for iv in ints:
            ng = iv["lims"][1] - iv["lims"][0] + 1
            start.append(off + 1)
            lvl = rng.uniform(-29.0, -26.5) if iv["dens"] else rng.uniform(-28.0, -25.0)
            if iv["id"] == "h2o_self":
                lvl = rng.uniform(-27.0, -25.0)
            g = np.linspace(0.0, 1.0, ng)[None, None, :]
            t = ((temp_ref - 250.0) / 100.0)[:, None, None]
            e = np.linspace(0.0, 1.0, NETA)[None, :, None]
            kmin[:, :, off:off + ng] = 10.0 ** (lvl + 2.0 * g - 0.4 * t + 0.3 * e)
            off += ng
        return ints, kmin, np.array(start, np.int32)

    ints_lo, kminor_lower, kstart_lo = minor_block(0)
    ints_up, kminor_upper, kstart_up = minor_block(1)

    def pack(ints):
        return dict(
            gases=[iv["id"] for iv in ints],
            lims=np.array([iv["lims"] for iv in ints], np.int32).reshape(-1, 2),
            dens=np.array([iv["dens"] for iv in ints], np.int32),
            sgas=[iv["sgas"] for iv in ints],
            comp=np.array([iv["comp"] for iv in ints], np.int32))

    lo, up = pack(ints_lo), pack(ints_up)

    d = dict(
        kind=kind, gas_names=list(gas_names), key_species=key_species,
        bnd_limits_gpt=band_lims_gpt,
        bnd_limits_wavenumber=np.array(wvn, np.float64),
        press_ref=press_ref, press_ref_trop=PRESS_REF_TROP, temp_ref=temp_ref,
        absorption_coefficient_ref_P=1013.25, absorption_coefficient_ref_T=273.15,
        vmr_ref=vmr_ref, kmajor=kmajor,
        kminor_lower=kminor_lower, kminor_upper=kminor_upper,
        gas_minor=list(_MINOR_GAS_DENSE if dense else _MINOR_GAS),
        identifier_minor=list(_MINOR_IDS_DENSE if dense else _MINOR_IDS),
        minor_gases_lower=lo["gases"], minor_gases_upper=up["gases"],
        minor_limits_gpt_lower=lo["lims"], minor_limits_gpt_upper=up["lims"],
        minor_scales_with_density_lower=lo["dens"], minor_scales_with_density_upper=up["dens"],
        scaling_gas_lower=lo["sgas"], scaling_gas_upper=up["sgas"],
        scale_by_complement_lower=lo["comp"], scale_by_complement_upper=up["comp"],
        kminor_start_lower=kstart_lo, kminor_start_upper=kstart_up,
    )

    if kind == "lw":
        tpl = np.linspace(temp_ref[0], temp_ref[-1], NPLANCK)
        totplnk = np.stack([_planck_band_radiance(a, b, tpl) for (a, b) in wvn])
        pf = rng.uniform(0.3, 1.0, (1, 1, 1, ngpt)) * (1.0 + 0.2 * np.sin(3.0 * tt + 2.0 * pp + ee + 5 * gfrac))
        pf = pf * np.ones((NTEMP, NPRES + 1, NETA, 1))
        pfr = pf.reshape(NTEMP, NPRES + 1, NETA, nband, ngpb)
        pfr = pfr / pfr.sum(axis=-1, keepdims=True)
        d["totplnk"] = np.ascontiguousarray(totplnk)
        d["plank_fraction"] = np.ascontiguousarray(pfr.reshape(NTEMP, NPRES + 1, NETA, ngpt))
        d["rayl_lower"] = None
        d["rayl_upper"] = None
    else:
        # Solar source per g-point: a 5778 K blackbody split over bands, random within band.
        frac = np.array([_planck_band_radiance(a, b, [5778.0])[0] for (a, b) in wvn])
        frac = frac / frac.sum()
        w = rng.uniform(0.5, 1.5, ngpt).reshape(nband, ngpb)
        w = w / w.sum(axis=1, keepdims=True)
        quiet = (1360.8 * frac[:, None] * w).reshape(-1)
        d["solar_source_quiet"] = quiet
        d["solar_source_facular"] = quiet * rng.uniform(0.5e-3, 2e-3, ngpt)
        d["solar_source_sunspot"] = -quiet * rng.uniform(1e-8, 5e-8, ngpt)
        d["tsi_default"] = 1360.858
        d["mg_default"] = 0.1567652
        d["sb_default"] = 902.8053
        nu_c = np.array([0.5 * (a + b) for (a, b) in wvn])
        ray = 4.02e-28 * (np.repeat(nu_c, ngpb) / 1.0e4) ** 4
        t2 = ((temp_ref - 250.0) / 100.0)[:, None, None]
        e2 = np.linspace(0.0, 1.0, NETA)[None, :, None]
        g2 = np.tile(np.linspace(0.0, 1.0, ngpb), nband)[None, None, :]
        var = 1.0 + 0.05 * np.sin(2.0 * np.pi * (e2 + t2 + 0.3 * g2))
        d["rayl_lower"] = np.ascontiguousarray(ray[None, None, :] * var)
        d["rayl_upper"] = np.ascontiguousarray(d["rayl_lower"] * 1.01)
    return d


def make_cloud_luts(kind: str, seed: int = 7):
    """Cloud optics LUTs in the reference file layout (Radiation_solver.cpp:286-329)."""
    rng = np.random.default_rng(seed + (0 if kind == "lw" else 50))
    wvn = LW_BAND_WVN if kind == "lw" else SW_BAND_WVN
    nband = len(wvn)
    nsl, nsi, nrgh = 20, 18, 3
    rl_lwr, rl_upr = 2.5, 21.5
    ri_lwr, ri_upr = 10.0, 180.0
    rel = np.linspace(rl_lwr, rl_upr, nsl)
    rei = np.linspace(ri_lwr, ri_upr, nsi)
    nu = np.array([0.5 * (a + b) for (a, b) in wvn])
    lam = 1.0e4 / nu  # um
    # Liquid: ext ~ 1.5 Qext / (rho r), rho = 1e6 g m-3 -> m2 g-1.
    x_l = 2 * np.pi * rel[None, :] / lam[:, None]
    qext_l = 2.0 - 4.0 / np.maximum(x_l, 0.5) * np.sin(np.minimum(x_l, 20.0) * 0.3) ** 2 * 0.3
    qext_l = np.clip(qext_l, 0.3, 2.6)
    ext_l = 1.5 * qext_l / (1.0e6 * rel[None, :] * 1.0e-6)
    if kind == "lw":
        ssa_l = np.clip(0.25 + 0.35 * np.tanh(rel[None, :] / 12.0) * (nu[:, None] / 3000.0 + 0.3), 0.05, 0.9)
    else:
        ssa_l = np.clip(1.0 - 1e-6 - 0.08 * (lam[:, None] / 3.0) ** 2 * (rel[None, :] / 10.0), 0.5, 1.0 - 1e-7)
    asy_l = np.clip(0.78 + 0.08 * np.tanh(rel[None, :] / 8.0) + 0.01 * rng.standard_normal((nband, nsl)), 0.5, 0.95)
    x_i = 2 * np.pi * rei[None, :] / lam[:, None]
    qext_i = np.clip(2.0 + 0.2 * np.sin(x_i * 0.05), 1.5, 2.5)
    ext_i0 = 1.5 * qext_i / (0.917e6 * rei[None, :] * 1.0e-6)
    if kind == "lw":
        ssa_i0 = np.clip(0.3 + 0.3 * np.tanh(rei[None, :] / 60.0) * (nu[:, None] / 3000.0 + 0.4), 0.05, 0.9)
    else:
        ssa_i0 = np.clip(1.0 - 1e-6 - 0.1 * (lam[:, None] / 3.0) ** 1.5 * (rei[None, :] / 50.0), 0.45, 1.0 - 1e-7)
    asy_i0 = np.clip(0.74 + 0.06 * np.tanh(rei[None, :] / 50.0) + 0.01 * rng.standard_normal((nband, nsi)), 0.5, 0.95)
    rough = np.array([0.97, 1.0, 1.03])[:, None, None]
    return dict(
        kind=kind,
        bnd_limits_wavenumber=np.array(wvn, np.float64),
        radliq_lwr=rl_lwr, radliq_upr=rl_upr, radliq_fac=1.0 / (rel[1] - rel[0]),
        radice_lwr=ri_lwr, radice_upr=ri_upr, radice_fac=1.0 / (rei[1] - rei[0]),
        lut_extliq=np.ascontiguousarray(ext_l), lut_ssaliq=np.ascontiguousarray(ssa_l),
        lut_asyliq=np.ascontiguousarray(asy_l),
        lut_extice=np.ascontiguousarray(ext_i0[None] * rough),
        lut_ssaice=np.ascontiguousarray(np.clip(ssa_i0[None] * rough ** 0.01, 0.0, 1.0 - 1e-7)),
        lut_asyice=np.ascontiguousarray(np.clip(asy_i0[None] * rough ** 0.2, 0.0, 0.99)),
    )


def make_aerosol_luts(seed: int = 11, nband: int = 14, nhum: int = 12, nphilic: int = 5, nphobic: int = 14):
    """Aerosol optics tables with the variables and dimension order that
    load_and_init_aerosol_optics reads (src_test/Radiation_solver.cu:366-401):
    relative_humidity2 (nhum, increasing, last 1), mass_ext/ssa/asymmetry_sw_hydrophobic
    (hydrophobic, band_sw) and _hydrophilic (hydrophilic, relative_humidity, band_sw).
    Hydrophilic extinction grows with humidity; mass extinction is in m2/kg."""
    rng = np.random.default_rng(seed)
    rh2 = np.concatenate([np.linspace(0.1, 0.9, nhum - 3), [0.95, 0.98, 1.0]])
    growth = (1.0 + 2.0 * rh2 ** 4)[None, :, None]
    return {
        "relative_humidity2": rh2,
        "mass_ext_sw_hydrophobic": rng.uniform(2.0e2, 6.0e3, (nphobic, nband)),
        "ssa_sw_hydrophobic": rng.uniform(0.6, 0.99, (nphobic, nband)),
        "asymmetry_sw_hydrophobic": rng.uniform(0.5, 0.8, (nphobic, nband)),
        "mass_ext_sw_hydrophilic": rng.uniform(1.0e3, 8.0e3, (nphilic, 1, nband)) * growth,
        "ssa_sw_hydrophilic": np.minimum(rng.uniform(0.85, 0.99, (nphilic, nhum, nband)), 1.0),
        "asymmetry_sw_hydrophilic": rng.uniform(0.6, 0.8, (nphilic, nhum, nband)),
    }


def make_aerosols(play: np.ndarray, seed: int = 12):
    """Mass mixing ratios aermr01 .. aermr11 (kg/kg, (nlay, ncol)) decaying with height, and a
    relative humidity field in [0, 1] (higher near the surface), for the layers of play."""
    rng = np.random.default_rng(seed)
    z = 7.0 * np.log(1.0e5 / play)   # km
    shape = np.exp(-z / 2.0)
    base = [2e-9, 8e-9, 1e-9, 5e-9, 1e-8, 4e-9, 3e-9, 2e-9, 5e-10, 5e-10, 6e-9]
    aer = {f"aermr{i + 1:02d}": base[i] * shape * rng.lognormal(0.0, 0.5, play.shape) for i in range(11)}
    rh = np.clip(0.2 + 0.7 * shape + rng.normal(0.0, 0.1, play.shape), 0.0, 1.0)
    return aer, rh


def make_atmosphere(ncol: int, nlay: int, seed: int = 42, clouds: bool = True,
                    nband_lw: int = 16, nband_sw: int = 14, top_at_1: bool = True, trace_gases: bool = False):
    """Synthetic atmosphere in the reference layouts (column fastest; numpy (nlay, ncol)).

    Pressure levels are log spaced from 1e5 Pa to the top (clamped to the table minimum);
    T = max(288 - 6.5 z[km], 200) + N(0, 2 K); h2o = 0.015 exp(-z / 2 km); o3 a Gaussian
    peak of 8e-6 at 25 km (5 km width); scalar co2, ch4, n2o, o2, n2.  Heights use
    z = H ln(1e5 / p) with H = 7 km.  Arrays are float64, shaped (nlay, ncol) so that the
    flat memory is the reference's column-fastest (ncol, nlay) Fortran array.
    """
    rng = np.random.default_rng(seed)
    plev1 = np.exp(np.linspace(np.log(1.0e5), np.log(P_TOP), nlay + 1))  # surface -> top
    plev1[-1] = P_TOP
    play1 = np.sqrt(plev1[1:] * plev1[:-1])
    if top_at_1:
        plev1 = plev1[::-1].copy()
        play1 = play1[::-1].copy()
    plev = np.repeat(plev1[:, None], ncol, axis=1)
    play = np.repeat(play1[:, None], ncol, axis=1)
    z = 7.0 * np.log(1.0e5 / play)  # km
    tlay = np.maximum(288.0 - 6.5 * z, 200.0) + rng.normal(0.0, 2.0, (nlay, ncol))
    tlev = np.empty((nlay + 1, ncol))
    tlev[1:-1] = 0.5 * (tlay[1:] + tlay[:-1])
    tlev[0] = 1.5 * tlay[0] - 0.5 * tlay[1]
    tlev[-1] = 1.5 * tlay[-1] - 0.5 * tlay[-2]
    tlev = np.clip(tlev, 161.0, 354.0)
    sfc_lev = nlay if top_at_1 else 0
    tsfc = tlev[sfc_lev].copy()
    h2o = 0.015 * np.exp(-z / 2.0)
    o3 = 8.0e-6 * np.exp(-((z - 25.0) / 5.0) ** 2)
    gases = {"h2o": h2o, "o3": o3, "co2": np.array([[4.0e-4]]), "ch4": np.array([[1.8e-6]]),
             "n2o": np.array([[3.2e-7]]), "o2": np.array([[0.2095]]), "n2": np.array([[0.7808]])}
    if trace_gases:   # scalar halocarbons, co and no2 (ATM_GASES_DENSE), drawn after every other field
        gases.update({g: np.array([[v]]) for g, v in _TRACE_VMR.items()})
    atm = dict(ncol=ncol, nlay=nlay, top_at_1=top_at_1, play=play, plev=plev, tlay=tlay,
               tlev=tlev, tsfc=tsfc, gases=gases,
               emis_sfc=np.full((ncol, nband_lw), 0.98),
               mu0=rng.uniform(0.1, 1.0, ncol),
               tsi_scaling=np.ones(ncol))
    alb = rng.uniform(0.05, 0.3, ncol)
    atm["sfc_alb_dir"] = np.repeat(alb[:, None], nband_sw, axis=1)
    atm["sfc_alb_dif"] = atm["sfc_alb_dir"].copy()
    lwp = np.zeros((nlay, ncol))
    iwp = np.zeros((nlay, ncol))
    rel = np.zeros((nlay, ncol))
    rei = np.zeros((nlay, ncol))
    if clouds:
        liq = (play > 5.0e4) & (play < 9.0e4) & (rng.random((nlay, ncol)) < 0.30)
        ice = (play > 1.5e4) & (play < 4.0e4) & (rng.random((nlay, ncol)) < 0.20)
        lwp[liq] = 50.0 * np.exp(rng.standard_normal(liq.sum()))
        iwp[ice] = 20.0 * np.exp(rng.standard_normal(ice.sum()))
        rel[liq] = rng.uniform(5.0, 15.0, liq.sum())
        rei[ice] = rng.uniform(20.0, 80.0, ice.sum())
    # Effective radii must lie inside the LUT even where no cloud is present.
    rel[rel == 0.0] = 10.0
    rei[rei == 0.0] = 50.0
    atm.update(lwp=lwp, iwp=iwp, rel=rel, rei=rei)
    return atm


def col_dry_from(h2o: np.ndarray, plev: np.ndarray) -> np.ndarray:
    """Dry-air column [molecules cm-2]; restates src/Gas_optics_rrtmgp.cpp:764-792."""
    g0, avogad, m_dry, m_h2o = 9.80665, 6.02214076e23, 0.028964, 0.018016
    dp = np.abs(plev[:-1] - plev[1:])
    m_air = (m_dry + m_h2o * h2o) / (1.0 + h2o)
    cd = 10.0 * dp * avogad / (1000.0 * m_air * 100.0 * g0)
    return cd / (1.0 + h2o)
