"""Column-radiation driver: the sequence of Radiation_solver_longwave/shortwave::solve_gpu
(src_test/Radiation_solver.cu:419-657, :683-950) over the C ABI.

LW: gas_optics -> cloud_optics (1scl) -> add_to by band -> rte_lw -> broadband reduce.
SW: gas_optics -> toa_src x tsi_scaling -> cloud_optics (2str) -> delta_scale -> add_to by
band -> rte_sw -> broadband reduce.  Both add heating rates.  Buffers are allocated once per
(ncol, nlay, dtype) and reused, so repeated solves launch kernels only.
"""
from __future__ import annotations

import torch

from . import api

ATM_KEYS_2D = ("play", "plev", "tlay", "tlev", "lwp", "iwp", "rel", "rei")


class Radiation_solver:
    def __init__(self, kdist_lw: dict, kdist_sw: dict, cloud_lw: dict | None, cloud_sw: dict | None,
                 available_gases, delta_cloud: bool = True, aerosol_sw: dict | None = None,
                 delta_aerosol: bool = False):
        self.klw = api.Gas_optics_rrtmgp(kdist_lw, available_gases)
        self.ksw = api.Gas_optics_rrtmgp(kdist_sw, available_gases)
        self.clw = api.Cloud_optics(cloud_lw) if cloud_lw is not None else None
        self.csw = api.Cloud_optics(cloud_sw) if cloud_sw is not None else None
        self.delta_cloud = delta_cloud
        # Aerosol_optics_gpu of Radiation_solver_shortwave (src_test/Radiation_solver.cu:664-680)
        self.aer = api.Aerosol_optics(aerosol_sw) if aerosol_sw is not None else None
        self.delta_aerosol = delta_aerosol
        self._bufs = {}

    def _buffers(self, key, like, ncol, nlay, kind):
        b = self._bufs.get((key, kind))
        if b is not None:
            return b
        dt, dev = like.dtype, like.device
        nlev = nlay + 1
        if kind == "lw":
            ng = self.klw.get_ngpt()
            b = {k: torch.empty((ng, nlay, ncol), dtype=dt, device=dev)
                 for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec")}
            b["sfc_src"] = torch.empty((ng, ncol), dtype=dt, device=dev)
            b["sfc_src_jac"] = torch.empty((ng, ncol), dtype=dt, device=dev)
            b["cloud_tau"] = torch.empty((self.klw.get_nband(), nlay, ncol), dtype=dt, device=dev)
            b["gpt_up"] = torch.empty((ng, nlev, ncol), dtype=dt, device=dev)
            b["gpt_dn"] = torch.empty((ng, nlev, ncol), dtype=dt, device=dev)
        else:
            ng = self.ksw.get_ngpt()
            b = {k: torch.empty((ng, nlay, ncol), dtype=dt, device=dev) for k in ("tau", "ssa", "g")}
            b["toa_src"] = torch.empty((ng, ncol), dtype=dt, device=dev)
            nb = self.ksw.get_nband()
            b.update({k: torch.empty((nb, nlay, ncol), dtype=dt, device=dev) for k in ("c_tau", "c_ssa", "c_g")})
            for k in ("gpt_up", "gpt_dn", "gpt_dir"):
                b[k] = torch.empty((ng, nlev, ncol), dtype=dt, device=dev)
            b["ws"] = api.Rte_sw.workspace(ncol, nlay, ng, like).clone()
            if dt == torch.float32 and nlay <= 128:
                # absorbed flux per (layer, g-point) for the heating rates (rte_sw_abs)
                b["gpt_abs"] = torch.empty((ng, nlay, ncol), dtype=dt, device=dev)
        for k in ("flux_up", "flux_dn", "flux_net", "flux_dn_dir"):
            b[k] = torch.empty((nlev, ncol), dtype=dt, device=dev)
        b["heating_rate"] = torch.empty((nlay, ncol), dtype=dt, device=dev)
        self._bufs[(key, kind)] = b
        return b

    def solve_lw(self, atm: dict, with_clouds: bool = True, top_at_1: bool = True):
        """atm: torch tensors play, plev, tlay, tlev (nlay[+1], ncol), tsfc (ncol), emis_sfc
        (ncol, nband), gases {name: tensor}, lwp/iwp/rel/rei (nlay, ncol)."""
        from . import _abi
        import ctypes as C
        play = atm["play"]
        nlay, ncol = play.shape
        key = (ncol, nlay, play.dtype)
        b = self._buffers(key, play, ncol, nlay, "lw")
        lib = _abi.load()
        sfx = api._sfx(play)
        s = api._stream()
        P = api._ptr
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
        _abi.check(getattr(lib, "rrtmgp_b200_gas_optics_lw" + sfx)(
            self.klw.handle, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]), P(atm["tsfc"]), P(atm["tlev"]),
            None, arr, len(atm["gases"]), P(b["tau"]), P(b["lay_src"]), P(b["lev_src_inc"]), P(b["lev_src_dec"]),
            P(b["sfc_src"]), P(b["sfc_src_jac"]), s))
        if with_clouds and self.clw is not None:
            _abi.check(getattr(lib, "rrtmgp_b200_cloud_optics_1scl" + sfx)(
                self.clw.handle, ncol, nlay, P(atm["lwp"]), P(atm["iwp"]), P(atm["rel"]), P(atm["rei"]),
                P(b["cloud_tau"]), s))
            _abi.check(getattr(lib, "rrtmgp_b200_add_to_1scl" + sfx)(
                self.klw.bands.handle, ncol, nlay, P(b["tau"]), P(b["cloud_tau"]), self.klw.get_nband(), s))
        _abi.check(getattr(lib, "rrtmgp_b200_rte_lw" + sfx)(
            self.klw.bands.handle, ncol, nlay, int(top_at_1), P(b["tau"]), P(b["lay_src"]), P(b["lev_src_inc"]),
            P(b["lev_src_dec"]), P(b["sfc_src"]), P(atm["emis_sfc"]), None, 1, P(b["gpt_up"]), P(b["gpt_dn"]), s))
        _abi.check(getattr(lib, "rrtmgp_b200_fluxes_broadband" + sfx)(
            ncol, nlay + 1, self.klw.get_ngpt(), P(b["gpt_up"]), P(b["gpt_dn"]), None, P(b["flux_up"]),
            P(b["flux_dn"]), None, P(b["flux_net"]), s))
        if play.dtype == torch.float32:
            # FP32: from per-layer absorbed flux (a difference of FP32 level fluxes loses ~1 K/day
            # in ~0.1 Pa top layers); FP64: the level-flux difference, exact to ~1e-9 K/day
            _abi.check(lib.rrtmgp_b200_heating_rate_lw_layers_f32(
                ncol, nlay, self.klw.get_ngpt(), int(top_at_1), P(b["tau"]), P(b["lay_src"]), P(b["lev_src_inc"]),
                P(b["lev_src_dec"]), P(b["gpt_up"]), P(b["gpt_dn"]), P(atm["plev"]), P(b["heating_rate"]), s))
        else:
            _abi.check(getattr(lib, "rrtmgp_b200_heating_rate" + sfx)(
                ncol, nlay, P(b["flux_up"]), P(b["flux_dn"]), P(atm["plev"]), P(b["heating_rate"]), s))
        return {k: b[k] for k in ("flux_up", "flux_dn", "flux_net", "heating_rate")}

    def solve_sw(self, atm: dict, with_clouds: bool = True, top_at_1: bool = True, with_aerosols: bool = False):
        """atm additionally needs mu0 (ncol), sfc_alb_dir / sfc_alb_dif (ncol, nband) and
        optionally tsi_scaling (ncol); with_aerosols: aerosols {aermr01 .. aermr11} and rh
        (nlay, ncol), their optics (delta-scaled if delta_aerosol) added by band after the
        clouds (switch_aerosol_optics, src_test/Radiation_solver.cu:794-807)."""
        from . import _abi
        play = atm["play"]
        nlay, ncol = play.shape
        key = (ncol, nlay, play.dtype)
        b = self._buffers(key, play, ncol, nlay, "sw")
        lib = _abi.load()
        sfx = api._sfx(play)
        s = api._stream()
        P = api._ptr
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
        _abi.check(getattr(lib, "rrtmgp_b200_gas_optics_sw" + sfx)(
            self.ksw.handle, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]), None, arr, len(atm["gases"]),
            P(b["tau"]), P(b["ssa"]), P(b["g"]), P(b["toa_src"]), s))
        if "tsi_scaling" in atm and atm["tsi_scaling"] is not None:
            b["toa_src"].mul_(atm["tsi_scaling"][None, :])
        nb = self.ksw.get_nband()
        if with_clouds and self.csw is not None:
            _abi.check(getattr(lib, "rrtmgp_b200_cloud_optics_2str" + sfx)(
                self.csw.handle, ncol, nlay, P(atm["lwp"]), P(atm["iwp"]), P(atm["rel"]), P(atm["rei"]),
                P(b["c_tau"]), P(b["c_ssa"]), P(b["c_g"]), s))
            if self.delta_cloud:
                _abi.check(getattr(lib, "rrtmgp_b200_delta_scale_2str" + sfx)(
                    ncol, nlay, nb, P(b["c_tau"]), P(b["c_ssa"]), P(b["c_g"]), s))
            _abi.check(getattr(lib, "rrtmgp_b200_add_to_2str" + sfx)(
                self.ksw.bands.handle, ncol, nlay, P(b["tau"]), P(b["ssa"]), P(b["g"]), P(b["c_tau"]),
                P(b["c_ssa"]), P(b["c_g"]), nb, s))
        if with_aerosols:
            assert self.aer is not None, "solver built without aerosol tables"
            a = self.aer.aerosol_optics(atm["aerosols"], atm["rh"], atm["plev"])
            if self.delta_aerosol:
                api.delta_scale(a["tau"], a["ssa"], a["g"])
            _abi.check(getattr(lib, "rrtmgp_b200_add_to_2str" + sfx)(
                self.ksw.bands.handle, ncol, nlay, P(b["tau"]), P(b["ssa"]), P(b["g"]), P(a["tau"]),
                P(a["ssa"]), P(a["g"]), nb, s))
        import ctypes as C
        if "gpt_abs" in b:
            # FP32 up to 128 layers: the solver also writes the flux each layer absorbs per g-point
            _abi.check(lib.rrtmgp_b200_rte_sw_abs_f32(
                self.ksw.bands.handle, ncol, nlay, int(top_at_1), P(b["tau"]), P(b["ssa"]), P(b["g"]),
                P(atm["mu0"]), P(b["toa_src"]), P(atm["sfc_alb_dir"]), P(atm["sfc_alb_dif"]), None, P(b["gpt_up"]),
                P(b["gpt_dn"]), P(b["gpt_dir"]), P(b["gpt_abs"]), s))
        else:
            _abi.check(getattr(lib, "rrtmgp_b200_rte_sw" + sfx)(
                self.ksw.bands.handle, ncol, nlay, int(top_at_1), P(b["tau"]), P(b["ssa"]), P(b["g"]), P(atm["mu0"]),
                P(b["toa_src"]), P(atm["sfc_alb_dir"]), P(atm["sfc_alb_dif"]), None, P(b["gpt_up"]), P(b["gpt_dn"]),
                P(b["gpt_dir"]), C.c_void_p(b["ws"].data_ptr()), C.c_size_t(b["ws"].numel()), s))
        _abi.check(getattr(lib, "rrtmgp_b200_fluxes_broadband" + sfx)(
            ncol, nlay + 1, self.ksw.get_ngpt(), P(b["gpt_up"]), P(b["gpt_dn"]), P(b["gpt_dir"]), P(b["flux_up"]),
            P(b["flux_dn"]), P(b["flux_dn_dir"]), P(b["flux_net"]), s))
        if "gpt_abs" in b:
            _abi.check(lib.rrtmgp_b200_heating_rate_from_layer_abs_f32(
                ncol, nlay, self.ksw.get_ngpt(), P(b["gpt_abs"]), P(atm["plev"]), P(b["heating_rate"]), s))
        elif play.dtype == torch.float32:   # as solve_lw
            _abi.check(lib.rrtmgp_b200_heating_rate_sw_layers_f32(
                ncol, nlay, self.ksw.get_ngpt(), int(top_at_1), P(b["tau"]), P(b["ssa"]), P(b["g"]), P(atm["mu0"]),
                P(b["gpt_up"]), P(b["gpt_dn"]), P(b["gpt_dir"]), P(atm["plev"]), P(b["heating_rate"]), s))
        else:
            _abi.check(getattr(lib, "rrtmgp_b200_heating_rate" + sfx)(
                ncol, nlay, P(b["flux_up"]), P(b["flux_dn"]), P(atm["plev"]), P(b["heating_rate"]), s))
        return {k: b[k] for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate")}


class Fused_solver:
    """FP32 column forward through the fused kernels (rrtmgp_b200_forward_lw_f32 / _sw_f32):
    same inputs and outputs as Radiation_solver.solve_lw / solve_sw, no g-point arrays."""

    def __init__(self, base: Radiation_solver, chunk: int = 0):
        self.base = base
        self.chunk = chunk
        self._out = {}

    def _outputs(self, kind, like, ncol, nlay):
        key = (kind, ncol, nlay, like.device)
        o = self._out.get(key)
        if o is None:
            o = {k: torch.empty((nlay + 1, ncol), dtype=torch.float32, device=like.device)
                 for k in ("flux_up", "flux_dn", "flux_net", "flux_dn_dir")}
            o["heating_rate"] = torch.empty((nlay, ncol), dtype=torch.float32, device=like.device)
            self._out[key] = o
        return o

    def solve_lw(self, atm: dict, with_clouds: bool = True):
        from . import _abi
        play = atm["play"]
        assert play.dtype == torch.float32, "the fused path is FP32"
        nlay, ncol = play.shape
        o = self._outputs("lw", play, ncol, nlay)
        P = api._ptr
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
        c = self.base.clw if (with_clouds and self.base.clw is not None) else None
        _abi.check(_abi.load().rrtmgp_b200_forward_lw_f32(
            self.base.klw.handle, c.handle if c else None, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]),
            P(atm["tlev"]), P(atm["tsfc"]), None, arr, len(atm["gases"]),
            P(atm["lwp"]) if c else None, P(atm["iwp"]) if c else None, P(atm["rel"]) if c else None,
            P(atm["rei"]) if c else None, P(atm["emis_sfc"]), P(o["flux_up"]), P(o["flux_dn"]), P(o["flux_net"]),
            P(o["heating_rate"]), int(self.chunk), api._stream()))
        return {k: o[k] for k in ("flux_up", "flux_dn", "flux_net", "heating_rate")}


    def solve_sw(self, atm: dict, with_clouds: bool = True, with_aerosols: bool = False):
        """with_aerosols: atm["aerosols"] {aermr01 .. aermr11} and atm["rh"] (nlay, ncol) through
        the base solver's aerosol tables, inside the fused kernel (rrtmgp_b200_forward_sw_aer_f32)."""
        from . import _abi
        play = atm["play"]
        assert play.dtype == torch.float32, "the fused path is FP32"
        nlay, ncol = play.shape
        o = self._outputs("sw", play, ncol, nlay)
        P = api._ptr
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
        c = self.base.csw if (with_clouds and self.base.csw is not None) else None
        tsi = atm.get("tsi_scaling")
        if with_aerosols:
            assert self.base.aer is not None, "solver built without aerosol tables"
            aer, keep_a = api.Gas_optics_rrtmgp._gases(atm["aerosols"], ncol, nlay, atm["play"])
            _abi.check(_abi.load().rrtmgp_b200_forward_sw_aer_f32(
                self.base.ksw.handle, c.handle if c else None, self.base.aer.handle, ncol, nlay, P(play),
                P(atm["plev"]), P(atm["tlay"]), None, arr, len(atm["gases"]), P(atm["lwp"]) if c else None,
                P(atm["iwp"]) if c else None, P(atm["rel"]) if c else None, P(atm["rei"]) if c else None,
                int(self.base.delta_cloud), aer, len(atm["aerosols"]), P(atm["rh"]), int(self.base.delta_aerosol),
                P(atm["mu0"]), P(tsi) if tsi is not None else None, P(atm["sfc_alb_dir"]), P(atm["sfc_alb_dif"]),
                P(o["flux_up"]), P(o["flux_dn"]), P(o["flux_dn_dir"]), P(o["flux_net"]), P(o["heating_rate"]),
                int(self.chunk), api._stream()))
            return {k: o[k] for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate")}
        _abi.check(_abi.load().rrtmgp_b200_forward_sw_f32(
            self.base.ksw.handle, c.handle if c else None, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]),
            None, arr, len(atm["gases"]), P(atm["lwp"]) if c else None, P(atm["iwp"]) if c else None,
            P(atm["rel"]) if c else None, P(atm["rei"]) if c else None, int(self.base.delta_cloud),
            P(atm["mu0"]), P(tsi) if tsi is not None else None, P(atm["sfc_alb_dir"]), P(atm["sfc_alb_dif"]),
            P(o["flux_up"]), P(o["flux_dn"]), P(o["flux_dn_dir"]), P(o["flux_net"]), P(o["heating_rate"]),
            int(self.chunk), api._stream()))
        return {k: o[k] for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate")}


def atm_to_device(atm: dict, dtype, device):
    """Convert a synthetic atmosphere (numpy, rrtmgp_b200.synthetic layout) to torch."""
    out = {}
    for k in ATM_KEYS_2D + ("tsfc", "mu0", "tsi_scaling", "emis_sfc", "sfc_alb_dir", "sfc_alb_dif"):
        out[k] = torch.as_tensor(atm[k], dtype=dtype, device=device).contiguous()
    out["gases"] = {k: torch.as_tensor(v.reshape(1) if v.size == 1 else v, dtype=dtype, device=device).contiguous()
                    for k, v in atm["gases"].items()}
    return out
