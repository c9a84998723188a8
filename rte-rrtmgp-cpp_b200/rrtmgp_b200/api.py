"""Python mirror of the reference's GPU class API over the C ABI.

Class and method names follow rte-rrtmgp-cpp (include/Gas_optics_rrtmgp.h, Cloud_optics.h,
Rte_lw.h, Rte_sw.h, Fluxes.h).  Arrays are torch CUDA tensors whose flat memory is the
reference's column-fastest Fortran layout, i.e. torch shapes are reversed:
(ncol, nlay) -> torch (nlay, ncol); (ncol, nlay, ngpt) -> torch (ngpt, nlay, ncol);
(nband, ncol) -> torch (ncol, nband).  float32 tensors run the FP32 kernels, float64 tensors
the FP64 instantiation.  Every call is asynchronous on torch's current stream.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi
from ._abi import check


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _sfx(t: torch.Tensor) -> str:
    if t.dtype == torch.float32:
        return "_f32"
    if t.dtype == torch.float64:
        return "_f64"
    raise TypeError(f"unsupported dtype {t.dtype}")


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("rrtmgp_b200 expects CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("rrtmgp_b200 expects contiguous tensors")
    return C.c_void_p(t.data_ptr())


def _call(name, dtype_tensor, *args):
    lib = _abi.load()
    return check(getattr(lib, "rrtmgp_b200_" + name + _sfx(dtype_tensor))(*args))


def _empty(shape, like):
    return torch.empty(shape, dtype=like.dtype, device=like.device)


def _release(fn, handle):
    """Destroy a native handle; a no-op once the interpreter has torn the modules down."""
    lib = getattr(_abi, "_lib", None) if _abi is not None else None
    if lib is not None and handle is not None:
        getattr(lib, fn)(handle)


class Bands:
    """Optical_props_gpu band/g-point discretisation (include/Optical_props.h:176-211)."""

    def __init__(self, handle, owner=None, band_lims=None):
        self.handle = handle
        self._owner = owner
        lib = _abi.load()
        nb, ng = C.c_int(), C.c_int()
        check(lib.rrtmgp_b200_bands_get(handle, C.byref(nb), C.byref(ng)))
        self.nband, self.ngpt = nb.value, ng.value

    @classmethod
    def from_limits(cls, band_lims_gpt):
        import numpy as np
        lims = np.ascontiguousarray(np.asarray(band_lims_gpt, np.int32))
        h = C.c_void_p()
        check(_abi.load().rrtmgp_b200_bands_create(len(lims), lims.ctypes.data_as(_abi.c_int_p), C.byref(h)))
        b = cls(h)
        b._own = True
        return b

    def __del__(self, _release=_release):
        if getattr(self, "_own", False):
            _release("rrtmgp_b200_bands_destroy", self.handle)


class Gas_optics_rrtmgp:
    """Gas_optics_rrtmgp_gpu: k-distribution gas optics (include/Gas_optics_rrtmgp.h:289-551)."""

    def __init__(self, tables: dict, available_gases):
        lib = _abi.load()
        t, keep = _abi.kdist_tables(tables)
        names, keep2 = _abi.string_array(list(available_gases))
        h = C.c_void_p()
        check(lib.rrtmgp_b200_kdist_create(C.byref(t), names, len(available_gases), C.byref(h)))
        self.handle = h
        info = _abi.KdistInfo()
        check(lib.rrtmgp_b200_kdist_get_info(h, C.byref(info)))
        self.info = info
        buf = C.create_string_buffer(64)
        self.gas_names = []
        for i in range(info.ngas):
            check(lib.rrtmgp_b200_kdist_gas_name(h, i, buf, 64))
            self.gas_names.append(buf.value.decode())
        self.bands = Bands(lib.rrtmgp_b200_kdist_bands(h), owner=self)
        self.band_lims_gpt = tables["bnd_limits_gpt"]

    def __del__(self, _release=_release):
        if getattr(self, "handle", None) is not None:
            _release("rrtmgp_b200_kdist_destroy", self.handle)
            self.handle = None

    def get_ngpt(self):
        return self.info.ngpt

    def get_nband(self):
        return self.info.nband

    def source_is_internal(self):
        return bool(self.info.is_longwave)

    def get_tsi(self):
        return self.info.tsi if not self.info.is_longwave else 0.0

    def set_solar_variability(self, mg_index, sb_index):
        lib = _abi.load()
        check(lib.rrtmgp_b200_kdist_set_solar_variability(self.handle, float(mg_index), float(sb_index)))
        info = _abi.KdistInfo()
        check(lib.rrtmgp_b200_kdist_get_info(self.handle, C.byref(info)))
        self.info = info

    @staticmethod
    def _gases(gases: dict, ncol, nlay, like):
        """GasConc array of the C ABI for {name: vmr}.  Every vmr must be a CUDA tensor on the
        device of `like` with its dtype (the kernel reads it as that type), shaped as a scalar,
        a profile (nlay,) / (nlay, 1) or a field (nlay, ncol); anything else raises before a
        pointer is taken."""
        arr = (_abi.GasConc * max(len(gases), 1))()
        keep = []
        for i, (name, v) in enumerate(gases.items()):
            if not isinstance(v, torch.Tensor):
                raise ValueError(f"gas '{name}': vmr must be a torch tensor")
            if v.dtype != like.dtype:
                raise ValueError(f"gas '{name}': vmr dtype {v.dtype} differs from the call's {like.dtype}")
            if v.dim() == 0 or v.numel() == 1:
                d1, d2 = 1, 1
            elif (v.dim() == 1 and v.shape[0] == nlay) or (v.dim() == 2 and v.shape == (nlay, 1)):
                d1, d2 = 1, nlay
            elif v.dim() == 2 and v.shape == (nlay, ncol):
                d1, d2 = ncol, nlay
            else:
                raise ValueError(f"gas '{name}': vmr shape {tuple(v.shape)} is none of (), ({nlay},), "
                                 f"({nlay}, 1), ({nlay}, {ncol})")
            if not v.is_cuda or v.device != like.device:
                raise ValueError(f"gas '{name}': vmr must be a CUDA tensor on {like.device}")
            v = v.contiguous()
            keep.append(v)
            arr[i].name = name.encode()
            arr[i].vmr = v.data_ptr()
            arr[i].dim1, arr[i].dim2 = d1, d2
        return arr, keep

    @staticmethod
    def get_col_dry(vmr_h2o, plev):
        nlay, ncol = vmr_h2o.shape
        out = _empty((nlay, ncol), plev)
        _call("get_col_dry", plev, ncol, nlay, _ptr(vmr_h2o), _ptr(plev), _ptr(out), _stream())
        return out

    def gas_optics_lw(self, play, plev, tlay, tsfc, gases: dict, tlev, col_dry=None):
        nlay, ncol = play.shape
        ng = self.info.ngpt
        arr, keep = self._gases(gases, ncol, nlay, play)
        out = {k: _empty((ng, nlay, ncol), play) for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec")}
        out["sfc_src"] = _empty((ng, ncol), play)
        out["sfc_src_jac"] = _empty((ng, ncol), play)
        _call("gas_optics_lw", play, self.handle, ncol, nlay, _ptr(play), _ptr(plev), _ptr(tlay), _ptr(tsfc),
              _ptr(tlev), _ptr(col_dry), arr, len(gases), _ptr(out["tau"]), _ptr(out["lay_src"]),
              _ptr(out["lev_src_inc"]), _ptr(out["lev_src_dec"]), _ptr(out["sfc_src"]),
              _ptr(out["sfc_src_jac"]), _stream())
        return out

    def gas_optics_sw(self, play, plev, tlay, gases: dict, col_dry=None):
        nlay, ncol = play.shape
        ng = self.info.ngpt
        arr, keep = self._gases(gases, ncol, nlay, play)
        out = {k: _empty((ng, nlay, ncol), play) for k in ("tau", "ssa", "g")}
        out["toa_src"] = _empty((ng, ncol), play)
        _call("gas_optics_sw", play, self.handle, ncol, nlay, _ptr(play), _ptr(plev), _ptr(tlay), _ptr(col_dry),
              arr, len(gases), _ptr(out["tau"]), _ptr(out["ssa"]), _ptr(out["g"]), _ptr(out["toa_src"]),
              _stream())
        return out

    def check_range(self, play, plev, tlay, tlev=None, tsfc=None, col_dry=None):
        nlay, ncol = play.shape
        _call("check_range", play, self.handle, ncol, nlay, _ptr(play), _ptr(plev), _ptr(tlay), _ptr(tlev),
              _ptr(tsfc), _ptr(col_dry), _stream())


class Cloud_optics:
    """Cloud_optics_gpu LUT cloud optics (include/Cloud_optics.h:80-131)."""

    def __init__(self, tables: dict):
        lib = _abi.load()
        t, keep = _abi.cloud_tables(tables)
        h = C.c_void_p()
        check(lib.rrtmgp_b200_cloud_create(C.byref(t), C.byref(h)))
        self.handle = h
        self.nband = t.nband

    def __del__(self, _release=_release):
        if getattr(self, "handle", None) is not None:
            _release("rrtmgp_b200_cloud_destroy", self.handle)
            self.handle = None

    def cloud_optics(self, clwp, ciwp, reliq, reice, two_stream=True):
        nlay, ncol = clwp.shape
        tau = _empty((self.nband, nlay, ncol), clwp)
        if two_stream:
            ssa, g = _empty(tau.shape, clwp), _empty(tau.shape, clwp)
            _call("cloud_optics_2str", clwp, self.handle, ncol, nlay, _ptr(clwp), _ptr(ciwp), _ptr(reliq),
                  _ptr(reice), _ptr(tau), _ptr(ssa), _ptr(g), _stream())
            return {"tau": tau, "ssa": ssa, "g": g}
        _call("cloud_optics_1scl", clwp, self.handle, ncol, nlay, _ptr(clwp), _ptr(ciwp), _ptr(reliq),
              _ptr(reice), _ptr(tau), _stream())
        return {"tau": tau}


AEROSOL_NAMES = tuple(f"aermr{i:02d}" for i in range(1, 12))


class Aerosol_optics:
    """Aerosol_optics_gpu band LUT aerosol optics (include/Aerosol_optics.h:64-86)."""

    def __init__(self, tables: dict):
        lib = _abi.load()
        t, keep = _abi.aerosol_tables(tables)
        h = C.c_void_p()
        check(lib.rrtmgp_b200_aerosol_create(C.byref(t), C.byref(h)))
        self.handle = h
        self.nband = t.nband

    def __del__(self, _release=_release):
        if getattr(self, "handle", None) is not None:
            _release("rrtmgp_b200_aerosol_destroy", self.handle)
            self.handle = None

    def aerosol_optics(self, aerosols: dict, rh, plev):
        """aerosols: {aermr01 .. aermr11: tensor (nlay, ncol), (nlay,) or scalar}; rh (nlay,
        ncol); plev (nlay+1, ncol).  Returns tau, ssa, g (nband, nlay, ncol)."""
        nlay, ncol = rh.shape
        arr, keep = Gas_optics_rrtmgp._gases(aerosols, ncol, nlay, rh)
        tau = _empty((self.nband, nlay, ncol), rh)
        ssa, g = _empty(tau.shape, rh), _empty(tau.shape, rh)
        _call("aerosol_optics", rh, self.handle, ncol, nlay, arr, len(aerosols), _ptr(rh), _ptr(plev), _ptr(tau),
              _ptr(ssa), _ptr(g), _stream())
        return {"tau": tau, "ssa": ssa, "g": g}


def delta_scale(tau, ssa, g):
    """Optical_props_2str_gpu::delta_scale, in place."""
    ngpt, nlay, ncol = tau.shape
    _call("delta_scale_2str", tau, ncol, nlay, ngpt, _ptr(tau), _ptr(ssa), _ptr(g), _stream())


def add_to(bands: Bands, inout: dict, inp: dict):
    """add_to(Optical_props_*_gpu&, const Optical_props_*_gpu&), in place on `inout`."""
    ngpt_in, nlay, ncol = inp["tau"].shape
    if "ssa" in inout:
        _call("add_to_2str", inout["tau"], bands.handle, ncol, nlay, _ptr(inout["tau"]), _ptr(inout["ssa"]),
              _ptr(inout["g"]), _ptr(inp["tau"]), _ptr(inp["ssa"]), _ptr(inp["g"]), ngpt_in, _stream())
    else:
        _call("add_to_1scl", inout["tau"], bands.handle, ncol, nlay, _ptr(inout["tau"]), _ptr(inp["tau"]),
              ngpt_in, _stream())


class Rte_lw:
    """Rte_lw_gpu::rte_lw (include/Rte_lw.h:65-73)."""

    @staticmethod
    def rte_lw(bands: Bands, tau, top_at_1, sources: dict, sfc_emis, inc_flux=None, n_gauss_angles=1,
               flux_up_jac=False):
        """Returns (up, dn), or (up, dn, up_jac) with flux_up_jac: the surface-temperature
        Jacobian of the upward g-point fluxes from sources["sfc_src_jac"] (the reference's
        do_jacobians output of lw_solver_noscat)."""
        ngpt, nlay, ncol = tau.shape
        up = _empty((ngpt, nlay + 1, ncol), tau)
        dn = _empty((ngpt, nlay + 1, ncol), tau)
        if flux_up_jac:
            jac = _empty((ngpt, nlay + 1, ncol), tau)
            _call("rte_lw_jac", tau, bands.handle, ncol, nlay, int(bool(top_at_1)), _ptr(tau),
                  _ptr(sources["lay_src"]), _ptr(sources["lev_src_inc"]), _ptr(sources["lev_src_dec"]),
                  _ptr(sources["sfc_src"]), _ptr(sources["sfc_src_jac"]), _ptr(sfc_emis), _ptr(inc_flux),
                  int(n_gauss_angles), _ptr(up), _ptr(dn), _ptr(jac), _stream())
            return up, dn, jac
        _call("rte_lw", tau, bands.handle, ncol, nlay, int(bool(top_at_1)), _ptr(tau), _ptr(sources["lay_src"]),
              _ptr(sources["lev_src_inc"]), _ptr(sources["lev_src_dec"]), _ptr(sources["sfc_src"]),
              _ptr(sfc_emis), _ptr(inc_flux), int(n_gauss_angles), _ptr(up), _ptr(dn), _stream())
        return up, dn


class Rte_sw:
    """Rte_sw_gpu::rte_sw (include/Rte_sw.h:65-75)."""

    _ws = {}

    @classmethod
    def workspace(cls, ncol, nlay, ngpt, like):
        nbytes = _abi.load().rrtmgp_b200_rte_sw_workspace_bytes(ncol, nlay, ngpt, int(like.dtype == torch.float64))
        key = (like.device, nbytes)
        ws = cls._ws.get(key)
        if ws is None:
            cls._ws.clear()
            ws = torch.empty(nbytes, dtype=torch.uint8, device=like.device)
            cls._ws[key] = ws
        return ws

    @classmethod
    def rte_sw(cls, bands: Bands, tau, ssa, g, top_at_1, mu0, inc_flux_dir, sfc_alb_dir, sfc_alb_dif,
               inc_flux_dif=None, workspace=None):
        ngpt, nlay, ncol = tau.shape
        up = _empty((ngpt, nlay + 1, ncol), tau)
        dn = _empty((ngpt, nlay + 1, ncol), tau)
        dr = _empty((ngpt, nlay + 1, ncol), tau)
        ws = workspace if workspace is not None else cls.workspace(ncol, nlay, ngpt, tau)
        _call("rte_sw", tau, bands.handle, ncol, nlay, int(bool(top_at_1)), _ptr(tau), _ptr(ssa), _ptr(g),
              _ptr(mu0), _ptr(inc_flux_dir), _ptr(sfc_alb_dir), _ptr(sfc_alb_dif), _ptr(inc_flux_dif),
              _ptr(up), _ptr(dn), _ptr(dr), C.c_void_p(ws.data_ptr()) if ws.numel() else None,
              C.c_size_t(ws.numel()), _stream())
        return up, dn, dr


class Fluxes_broadband:
    """Fluxes_broadband_gpu::reduce (include/Fluxes.h:151-162)."""

    @staticmethod
    def reduce(gpt_flux_up, gpt_flux_dn, gpt_flux_dn_dir=None):
        ngpt, nlev, ncol = gpt_flux_up.shape
        out = {k: _empty((nlev, ncol), gpt_flux_up) for k in ("flux_up", "flux_dn", "flux_net")}
        out["flux_dn_dir"] = _empty((nlev, ncol), gpt_flux_up) if gpt_flux_dn_dir is not None else None
        _call("fluxes_broadband", gpt_flux_up, ncol, nlev, ngpt, _ptr(gpt_flux_up), _ptr(gpt_flux_dn),
              _ptr(gpt_flux_dn_dir), _ptr(out["flux_up"]), _ptr(out["flux_dn"]), _ptr(out["flux_dn_dir"]),
              _ptr(out["flux_net"]), _stream())
        return out


class Fluxes_byband:
    """Fluxes_byband_gpu::reduce (include/Fluxes.h:186-211), band sums as the F90 kernel."""

    @staticmethod
    def reduce(bands: Bands, gpt_flux_up, gpt_flux_dn, gpt_flux_dn_dir=None):
        ngpt, nlev, ncol = gpt_flux_up.shape
        nb = bands.nband
        out = {k: _empty((nb, nlev, ncol), gpt_flux_up) for k in ("bnd_flux_up", "bnd_flux_dn", "bnd_flux_net")}
        out["bnd_flux_dn_dir"] = _empty((nb, nlev, ncol), gpt_flux_up) if gpt_flux_dn_dir is not None else None
        _call("fluxes_byband", gpt_flux_up, bands.handle, ncol, nlev, _ptr(gpt_flux_up), _ptr(gpt_flux_dn),
              _ptr(gpt_flux_dn_dir), _ptr(out["bnd_flux_up"]), _ptr(out["bnd_flux_dn"]),
              _ptr(out["bnd_flux_dn_dir"]), _ptr(out["bnd_flux_net"]), _stream())
        return out


def heating_rate(flux_up, flux_dn, plev):
    nlev, ncol = flux_up.shape
    hr = _empty((nlev - 1, ncol), flux_up)
    _call("heating_rate", flux_up, ncol, nlev - 1, _ptr(flux_up), _ptr(flux_dn), _ptr(plev), _ptr(hr), _stream())
    return hr
