"""ORACLE -- test infrastructure only.

numpy/ctypes front end of the FP64 C++ restatement in oracle/rrtmgp_oracle.cpp (built into
oracle/_build/liboracle.so by oracle/Makefile).  Arrays follow the same conventions as the
product's Python binding: numpy shapes are the reversed reference shapes
((ncol, nlay) -> (nlay, ncol), (ncol, nlay, ngpt) -> (ngpt, nlay, ncol), (nband, ncol) ->
(ncol, nband)), float64, C contiguous.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from rrtmgp_b200 import _abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
        _lib.oracle_last_error.restype = C.c_char_p
        _lib.oracle_kdist_create.argtypes = [C.POINTER(_abi.KdistTables), _abi.c_char_pp, C.c_int, C.POINTER(C.c_void_p)]
        _lib.oracle_cloud_create.argtypes = [C.POINTER(_abi.CloudTables), C.POINTER(C.c_void_p)]
        for name in ("oracle_kdist_destroy", "oracle_cloud_destroy"):
            getattr(_lib, name).argtypes = [C.c_void_p]
            getattr(_lib, name).restype = None
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_D)


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def set_threads(n: int):
    load().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return load().oracle_num_threads()


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"oracle status {status}: {msg}")
        self.status = status


def _check(st):
    if st != 0:
        raise OracleError(st, load().oracle_last_error().decode())


class GasOptics:
    def __init__(self, tables: dict, available_gases):
        lib = load()
        t, self._keep = _abi.kdist_tables(tables)
        names, self._keep2 = _abi.string_array(list(available_gases))
        h = C.c_void_p()
        _check(lib.oracle_kdist_create(C.byref(t), names, len(available_gases), C.byref(h)))
        self.h = h
        dims = (C.c_int * 8)()
        lib.oracle_kdist_dims(h, dims)
        self.ngas, self.nflav, self.nband, self.ngpt, self.nminor_lower, self.nminor_upper, self.idx_h2o = dims[:7]
        self.band_lims = np.ascontiguousarray(np.asarray(tables["bnd_limits_gpt"], np.int32))
        self.kind = tables.get("kind")

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.oracle_kdist_destroy(self.h)
            self.h = None

    def _gases(self, gases: dict):
        arr = (_abi.GasConc * max(len(gases), 1))()
        keep = []
        for i, (name, v) in enumerate(gases.items()):
            v = _f(v)
            keep.append(v)
            if v.size == 1:
                d1, d2 = 1, 1
            elif v.ndim == 1 or (v.ndim == 2 and v.shape[1] == 1):
                d1, d2 = 1, v.shape[0]
            else:
                d1, d2 = v.shape[1], v.shape[0]
            arr[i].name = name.encode()
            arr[i].vmr = v.ctypes.data
            arr[i].dim1, arr[i].dim2 = d1, d2
        return arr, keep

    def solar_source(self):
        out = np.empty(self.ngpt)
        load().oracle_kdist_solar_source(self.h, _p(out))
        return out

    def set_solar_variability(self, mg_index, sb_index):
        """Gas_optics_rrtmgp::set_solar_variability (src/Gas_optics_rrtmgp.cpp:745-760)."""
        lib = load()
        lib.oracle_kdist_set_solar_variability.argtypes = [C.c_void_p, C.c_double, C.c_double]
        st = lib.oracle_kdist_set_solar_variability(self.h, float(mg_index), float(sb_index))
        if st != 0:
            raise RuntimeError(lib.oracle_last_error().decode())

    def gas_optics_lw(self, play, plev, tlay, tsfc, gases, tlev, col_dry=None):
        play, plev, tlay, tsfc, tlev = map(_f, (play, plev, tlay, tsfc, tlev))
        col_dry = None if col_dry is None else _f(col_dry)
        nlay, ncol = play.shape
        arr, keep = self._gases(gases)
        out = {k: np.empty((self.ngpt, nlay, ncol)) for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec")}
        out["sfc_src"] = np.empty((self.ngpt, ncol))
        out["sfc_src_jac"] = np.empty((self.ngpt, ncol))
        _check(load().oracle_gas_optics_lw(self.h, ncol, nlay, _p(play), _p(plev), _p(tlay), _p(tsfc), _p(tlev),
                                           _p(col_dry), arr, len(gases), _p(out["tau"]), _p(out["lay_src"]),
                                           _p(out["lev_src_inc"]), _p(out["lev_src_dec"]), _p(out["sfc_src"]),
                                           _p(out["sfc_src_jac"])))
        return out

    def gas_optics_sw(self, play, plev, tlay, gases, col_dry=None):
        play, plev, tlay = map(_f, (play, plev, tlay))
        col_dry = None if col_dry is None else _f(col_dry)
        nlay, ncol = play.shape
        arr, keep = self._gases(gases)
        out = {k: np.empty((self.ngpt, nlay, ncol)) for k in ("tau", "ssa", "g")}
        out["toa_src"] = np.empty((self.ngpt, ncol))
        _check(load().oracle_gas_optics_sw(self.h, ncol, nlay, _p(play), _p(plev), _p(tlay), _p(col_dry), arr,
                                           len(gases), _p(out["tau"]), _p(out["ssa"]), _p(out["g"]),
                                           _p(out["toa_src"])))
        return out


def get_col_dry(h2o, plev):
    h2o, plev = _f(h2o), _f(plev)
    nlay, ncol = h2o.shape
    out = np.empty((nlay, ncol))
    load().oracle_get_col_dry(ncol, nlay, _p(h2o), _p(plev), _p(out))
    return out


class CloudOptics:
    def __init__(self, tables: dict):
        lib = load()
        t, self._keep = _abi.cloud_tables(tables)
        h = C.c_void_p()
        _check(lib.oracle_cloud_create(C.byref(t), C.byref(h)))
        self.h = h
        self.nband = t.nband

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.oracle_cloud_destroy(self.h)
            self.h = None

    def cloud_optics(self, clwp, ciwp, reliq, reice, two_stream=True):
        clwp, ciwp, reliq, reice = map(_f, (clwp, ciwp, reliq, reice))
        nlay, ncol = clwp.shape
        tau = np.empty((self.nband, nlay, ncol))
        ssa = np.empty_like(tau) if two_stream else None
        g = np.empty_like(tau) if two_stream else None
        _check(load().oracle_cloud_optics(self.h, ncol, nlay, _p(clwp), _p(ciwp), _p(reliq), _p(reice),
                                          int(two_stream), _p(tau), _p(ssa), _p(g)))
        return {"tau": tau, "ssa": ssa, "g": g} if two_stream else {"tau": tau}


AEROSOL_NAMES = tuple(f"aermr{i:02d}" for i in range(1, 12))


def aerosol_optics(tables: dict, aerosols: dict, rh, plev):
    """Aerosol optics (rrtmgp_oracle.cpp: oracle_aerosol_optics).  aerosols: aermr01 ..
    aermr11, each (nlay, ncol), (nlay,) or scalar; rh (nlay, ncol); plev (nlay+1, ncol)."""
    rh, plev = _f(rh), _f(plev)
    nlay, ncol = rh.shape
    ph = _f(tables["mass_ext_sw_hydrophobic"])
    pl = _f(tables["mass_ext_sw_hydrophilic"])
    nphobic, nband = ph.shape
    nphilic, nhum = pl.shape[0], pl.shape[1]
    fields = []
    for name in AEROSOL_NAMES:
        v = np.asarray(aerosols[name], dtype=np.float64)
        if v.size == 1:
            v = np.full((nlay, ncol), float(v.reshape(-1)[0]))
        elif v.ndim == 1 or v.shape[-1] == 1:
            v = np.repeat(v.reshape(nlay, 1), ncol, axis=1)
        fields.append(_f(v))
    ptrs = (_D * 11)(*[_p(f) for f in fields])
    tau = np.empty((nband, nlay, ncol))
    ssa, g = np.empty_like(tau), np.empty_like(tau)
    keep = [_f(tables[k]) for k in ("relative_humidity2", "ssa_sw_hydrophobic", "asymmetry_sw_hydrophobic",
                                    "ssa_sw_hydrophilic", "asymmetry_sw_hydrophilic")]
    load().oracle_aerosol_optics(nband, nhum, nphilic, nphobic, _p(keep[0]), _p(ph), _p(keep[1]), _p(keep[2]),
                                 _p(pl), _p(keep[3]), _p(keep[4]), ncol, nlay, ptrs, _p(rh), _p(plev), _p(tau),
                                 _p(ssa), _p(g))
    return {"tau": tau, "ssa": ssa, "g": g}


def delta_scale(tau, ssa, g):
    load().oracle_delta_scale(int(tau.size), _p(tau), _p(ssa), _p(g))


def add_to(band_lims, inout: dict, inp: dict):
    ngpt, nlay, ncol = inout["tau"].shape
    ngpt_in = inp["tau"].shape[0]
    two = "ssa" in inout and inout.get("ssa") is not None
    bl = None
    nband = 0
    if ngpt_in != ngpt:
        bl = np.ascontiguousarray(np.asarray(band_lims, np.int32))
        nband = len(bl)
        assert ngpt_in == nband
    load().oracle_add_to(ncol, nlay, ngpt, int(two), _p(inout["tau"]), _p(inout.get("ssa")), _p(inout.get("g")),
                         _p(_f(inp["tau"])), _p(_f(inp["ssa"])) if two else None,
                         _p(_f(inp["g"])) if two else None, nband, None if bl is None else bl.ctypes.data_as(_I))


def rte_lw(band_lims, tau, top_at_1, sources, sfc_emis, inc_flux=None, n_gauss_angles=1, flux_up_jac=False):
    """(up, dn), or (up, dn, up_jac) with flux_up_jac (surface-temperature Jacobian from
    sources["sfc_src_jac"])."""
    bl = np.ascontiguousarray(np.asarray(band_lims, np.int32))
    tau = _f(tau)
    ngpt, nlay, ncol = tau.shape
    up = np.empty((ngpt, nlay + 1, ncol))
    dn = np.empty_like(up)
    jac = np.empty_like(up) if flux_up_jac else None
    s = {k: _f(v) for k, v in sources.items() if v is not None}
    _check(load().oracle_rte_lw(ncol, nlay, ngpt, len(bl), bl.ctypes.data_as(_I), int(bool(top_at_1)), _p(tau),
                                _p(s["lay_src"]), _p(s["lev_src_inc"]), _p(s["lev_src_dec"]), _p(s["sfc_src"]),
                                _p(_f(sfc_emis)), None if inc_flux is None else _p(_f(inc_flux)),
                                int(n_gauss_angles), _p(up), _p(dn), _p(s["sfc_src_jac"]) if flux_up_jac else None,
                                _p(jac)))
    return (up, dn, jac) if flux_up_jac else (up, dn)


def rte_sw(band_lims, tau, ssa, g, top_at_1, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif, inc_flux_dif=None):
    bl = np.ascontiguousarray(np.asarray(band_lims, np.int32))
    tau, ssa, g = _f(tau), _f(ssa), _f(g)
    ngpt, nlay, ncol = tau.shape
    up = np.empty((ngpt, nlay + 1, ncol))
    dn = np.empty_like(up)
    dr = np.empty_like(up)
    _check(load().oracle_rte_sw(ncol, nlay, ngpt, len(bl), bl.ctypes.data_as(_I), int(bool(top_at_1)), _p(tau),
                                _p(ssa), _p(g), _p(_f(mu0)), _p(_f(inc_flux_dir)), _p(_f(sfc_alb_dir)),
                                _p(_f(sfc_alb_dif)), None if inc_flux_dif is None else _p(_f(inc_flux_dif)),
                                _p(up), _p(dn), _p(dr)))
    return up, dn, dr


def fluxes_broadband(up, dn, dn_dir=None):
    up, dn = _f(up), _f(dn)
    ngpt, nlev, ncol = up.shape
    out = {k: np.empty((nlev, ncol)) for k in ("flux_up", "flux_dn", "flux_net")}
    out["flux_dn_dir"] = np.empty((nlev, ncol)) if dn_dir is not None else None
    load().oracle_fluxes_broadband(ncol, nlev, ngpt, _p(up), _p(dn), None if dn_dir is None else _p(_f(dn_dir)),
                                   _p(out["flux_up"]), _p(out["flux_dn"]), _p(out["flux_dn_dir"]),
                                   _p(out["flux_net"]))
    return out


def fluxes_byband(band_lims, up, dn, dn_dir=None):
    bl = np.ascontiguousarray(np.asarray(band_lims, np.int32))
    up, dn = _f(up), _f(dn)
    ngpt, nlev, ncol = up.shape
    nb = len(bl)
    out = {k: np.empty((nb, nlev, ncol)) for k in ("bnd_flux_up", "bnd_flux_dn", "bnd_flux_net")}
    out["bnd_flux_dn_dir"] = np.empty((nb, nlev, ncol)) if dn_dir is not None else None
    load().oracle_fluxes_byband(ncol, nlev, nb, bl.ctypes.data_as(_I), _p(up), _p(dn),
                                None if dn_dir is None else _p(_f(dn_dir)), _p(out["bnd_flux_up"]),
                                _p(out["bnd_flux_dn"]), _p(out["bnd_flux_dn_dir"]), _p(out["bnd_flux_net"]))
    return out


def heating_rate(up, dn, plev):
    up, dn, plev = _f(up), _f(dn), _f(plev)
    nlev, ncol = up.shape
    hr = np.empty((nlev - 1, ncol))
    load().oracle_heating_rate(ncol, nlev - 1, _p(up), _p(dn), _p(plev), _p(hr))
    return hr


def forward_lw(kd: GasOptics, cloud: CloudOptics | None, atm: dict, col_dry=None):
    """Reference LW sequence of Radiation_solver_longwave::solve_gpu
    (src_test/Radiation_solver.cu:419-657): gas optics -> cloud 1scl added by band ->
    rte_lw -> broadband reduce, plus heating rates."""
    gases = atm["gases"]
    go = kd.gas_optics_lw(atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], gases, atm["tlev"], col_dry)
    if cloud is not None:
        c = cloud.cloud_optics(atm["lwp"], atm["iwp"], atm["rel"], atm["rei"], two_stream=False)
        add_to(kd.band_lims, {"tau": go["tau"]}, c)
    up, dn = rte_lw(kd.band_lims, go["tau"], atm["top_at_1"], go, atm["emis_sfc"])
    fl = fluxes_broadband(up, dn)
    fl["heating_rate"] = heating_rate(fl["flux_up"], fl["flux_dn"], atm["plev"])
    return fl


def forward_sw(kd: GasOptics, cloud: CloudOptics | None, atm: dict, col_dry=None, delta_cloud=True,
               aerosol_tables: dict | None = None, delta_aerosol=False):
    """Reference SW sequence of Radiation_solver_shortwave::solve_gpu
    (src_test/Radiation_solver.cu:683-950): gas optics, toa_src x tsi_scaling, cloud 2str +
    delta-scale added by band, aerosol optics (+ delta-scale) added by band when
    aerosol_tables is given (atm["aerosols"], atm["rh"]), rte_sw, broadband reduce, plus
    heating rates."""
    go = kd.gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"], col_dry)
    toa = go["toa_src"] * _f(atm["tsi_scaling"])[None, :]
    if cloud is not None:
        c = cloud.cloud_optics(atm["lwp"], atm["iwp"], atm["rel"], atm["rei"], two_stream=True)
        if delta_cloud:
            delta_scale(c["tau"], c["ssa"], c["g"])
        add_to(kd.band_lims, go, c)
    if aerosol_tables is not None:
        a = aerosol_optics(aerosol_tables, atm["aerosols"], atm["rh"], atm["plev"])
        if delta_aerosol:
            delta_scale(a["tau"], a["ssa"], a["g"])
        add_to(kd.band_lims, go, a)
    up, dn, dr = rte_sw(kd.band_lims, go["tau"], go["ssa"], go["g"], atm["top_at_1"], atm["mu0"], toa,
                        atm["sfc_alb_dir"], atm["sfc_alb_dif"])
    fl = fluxes_broadband(up, dn, dr)
    fl["heating_rate"] = heating_rate(fl["flux_up"], fl["flux_dn"], atm["plev"])
    return fl
