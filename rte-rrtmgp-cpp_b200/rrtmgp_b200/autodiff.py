"""Differentiable column radiation: torch.autograd.Function wrappers of the fused FP32
forward kernels whose backward calls the hand-written adjoint kernels through the C ABI
(rrtmgp_b200_adjoint_lw_f32, rrtmgp_b200_adjoint_sw_f32).

    out = longwave(fused_solver, atm)            # dict of flux_up, flux_dn, flux_net, heating_rate
    loss = (out["heating_rate"] * w).sum()
    loss.backward()                              # atm["tlay"].grad, atm["gases"]["h2o"].grad, ...

Differentiable inputs: longwave -- tlay, tlev, tsfc, the h2o and o3 volume mixing ratios
and (with clouds) lwp, iwp, rel, rei; shortwave -- tlay, h2o, o3, lwp, iwp, rel, rei and the
surface albedos.  Pressures, emissivity, mu0 and the other gases are constants.  The
backward recomputes the optical properties on chip (nothing of the forward is kept but its
inputs), so memory does not grow with the number of g-points.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _abi, api

_DIFF_KEYS = ("tlay", "tlev", "tsfc", "h2o", "o3", "lwp", "iwp", "rel", "rei")


def _reduce_to(grad, like):
    """Sum a (nlay, ncol) field gradient down to the shape of a scalar / profile input."""
    if grad is None or like is None:
        return None
    if like.numel() == grad.numel():
        return grad.reshape(like.shape)
    if like.numel() == 1:
        return grad.sum().reshape(like.shape)
    return grad.sum(dim=1).reshape(like.shape)   # profile: one value per layer


class _LongwaveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fused, static, tlay, tlev, tsfc, h2o, o3, lwp, iwp, rel, rei):
        atm = dict(static)
        atm.update(tlay=tlay, tlev=tlev, tsfc=tsfc, lwp=lwp, iwp=iwp, rel=rel, rei=rei)
        gases = dict(static["gases"])
        gases["h2o"], gases["o3"] = h2o, o3
        atm["gases"] = gases
        clouds = lwp is not None
        out = fused.solve_lw(atm, with_clouds=clouds)
        res = tuple(out[k].clone() for k in ("flux_up", "flux_dn", "flux_net", "heating_rate"))
        ctx.fused, ctx.atm, ctx.clouds = fused, atm, clouds
        ctx.save_for_backward(tlay, tlev, tsfc, h2o, o3)
        return res

    @staticmethod
    def backward(ctx, g_up, g_dn, g_net, g_hr):
        atm, fused = ctx.atm, ctx.fused
        play = atm["play"]
        nlay, ncol = play.shape
        dev = play.device

        def seed(g):
            return None if g is None else g.float().contiguous()

        up, dn, net = seed(g_up), seed(g_dn), seed(g_net)
        if net is not None:
            up = -net if up is None else up - net
            dn = net if dn is None else dn + net
        hr = seed(g_hr)
        grads = {k: torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
                 for k in ("tlay", "h2o", "o3", "lwp", "iwp", "rel", "rei")}
        grads["tlev"] = torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev)
        grads["tsfc"] = torch.empty((ncol,), dtype=torch.float32, device=dev)
        P = api._ptr
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
        c = fused.base.clw if ctx.clouds else None
        cl = (lambda k: P(atm[k])) if c else (lambda k: None)
        _abi.check(_abi.load().rrtmgp_b200_adjoint_lw_f32(
            fused.base.klw.handle, c.handle if c else None, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]),
            P(atm["tlev"]), P(atm["tsfc"]), None, arr, len(atm["gases"]), cl("lwp"), cl("iwp"), cl("rel"),
            cl("rei"), P(atm["emis_sfc"]), P(up), P(dn), P(hr), P(grads["tlay"]), P(grads["tlev"]),
            P(grads["tsfc"]), P(grads["h2o"]), P(grads["o3"]), P(grads["lwp"]) if c else None,
            P(grads["iwp"]) if c else None, P(grads["rel"]) if c else None, P(grads["rei"]) if c else None,
            0, api._stream()))
        tlay, tlev, tsfc, h2o, o3 = ctx.saved_tensors
        out = [None, None, grads["tlay"], grads["tlev"], grads["tsfc"], _reduce_to(grads["h2o"], h2o),
               _reduce_to(grads["o3"], o3)]
        out += [grads[k] if ctx.clouds else None for k in ("lwp", "iwp", "rel", "rei")]
        return tuple(out)


def longwave(fused, atm: dict, with_clouds: bool = True):
    """Differentiable fused FP32 longwave solve.  atm as for Fused_solver.solve_lw; its
    tlay, tlev, tsfc, gases["h2o"], gases["o3"], lwp, iwp, rel, rei may require grad."""
    clouds = with_clouds and fused.base.clw is not None
    static = {k: v for k, v in atm.items() if k not in _DIFF_KEYS}
    static["gases"] = {k: v for k, v in atm["gases"].items()}
    up, dn, net, hr = _LongwaveFn.apply(
        fused, static, atm["tlay"], atm["tlev"], atm["tsfc"], atm["gases"]["h2o"], atm["gases"]["o3"],
        atm["lwp"] if clouds else None, atm["iwp"] if clouds else None, atm["rel"] if clouds else None,
        atm["rei"] if clouds else None)
    return {"flux_up": up, "flux_dn": dn, "flux_net": net, "heating_rate": hr}


def adjoint_lw(fused, atm: dict, seed_up=None, seed_dn=None, seed_hr=None, with_clouds: bool = True, chunk: int = 0,
               with_fluxes: bool = False):
    """Direct call of the longwave adjoint: dict of gradients of
    sum(seed_up * flux_up + seed_dn * flux_dn + seed_hr * heating_rate).  with_fluxes: one
    launch that also returns the forward fluxes (rrtmgp_b200_forward_adjoint_lw_f32), as
    (fluxes, gradients)."""
    play = atm["play"]
    nlay, ncol = play.shape
    dev = play.device
    c = fused.base.clw if (with_clouds and fused.base.clw is not None) else None
    grads = {k: torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
             for k in ("tlay", "h2o", "o3", "lwp", "iwp", "rel", "rei")}
    grads["tlev"] = torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev)
    grads["tsfc"] = torch.empty((ncol,), dtype=torch.float32, device=dev)
    P = api._ptr
    arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
    cl = (lambda k: P(atm[k])) if c else (lambda k: None)
    args = [fused.base.klw.handle, c.handle if c else None, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]),
            P(atm["tlev"]), P(atm["tsfc"]), None, arr, len(atm["gases"]), cl("lwp"), cl("iwp"), cl("rel"),
            cl("rei"), P(atm["emis_sfc"]), P(seed_up), P(seed_dn), P(seed_hr), P(grads["tlay"]), P(grads["tlev"]),
            P(grads["tsfc"]), P(grads["h2o"]), P(grads["o3"]), P(grads["lwp"]) if c else None,
            P(grads["iwp"]) if c else None, P(grads["rel"]) if c else None, P(grads["rei"]) if c else None]
    if not with_fluxes:
        _abi.check(_abi.load().rrtmgp_b200_adjoint_lw_f32(*args, int(chunk), api._stream()))
        return grads
    fl = {k: torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev) for k in ("flux_up", "flux_dn", "flux_net")}
    fl["heating_rate"] = torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
    _abi.check(_abi.load().rrtmgp_b200_forward_adjoint_lw_f32(
        *args, P(fl["flux_up"]), P(fl["flux_dn"]), P(fl["flux_net"]), P(fl["heating_rate"]), int(chunk),
        api._stream()))
    return fl, grads


def adjoint_sw(fused, atm: dict, seed_up=None, seed_dn=None, seed_dir=None, seed_hr=None, with_clouds: bool = True,
               with_fluxes: bool = False, with_aerosols: bool = False):
    """Direct call of the shortwave adjoint: dict of gradients of sum(seed_up * flux_up +
    seed_dn * flux_dn + seed_dir * flux_dn_dir + seed_hr * heating_rate) w.r.t. tlay, h2o, o3,
    lwp, iwp, rel, rei (nlay, ncol) and sfc_alb_dir, sfc_alb_dif (ncol, nband).  with_fluxes:
    one launch that also returns the forward fluxes (rrtmgp_b200_forward_adjoint_sw_f32), as
    (fluxes, gradients).  with_aerosols: atm["aerosols"] and atm["rh"] through the base
    solver's aerosol tables in the recomputed forward (rrtmgp_b200_forward_adjoint_sw_aer_f32)."""
    play = atm["play"]
    nlay, ncol = play.shape
    dev = play.device
    c = fused.base.csw if (with_clouds and fused.base.csw is not None) else None
    nb = fused.base.ksw.get_nband()
    grads = {k: torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
             for k in ("tlay", "h2o", "o3", "lwp", "iwp", "rel", "rei")}
    grads["sfc_alb_dir"] = torch.empty((ncol, nb), dtype=torch.float32, device=dev)
    grads["sfc_alb_dif"] = torch.empty((ncol, nb), dtype=torch.float32, device=dev)
    P = api._ptr
    arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
    cl = (lambda k: P(atm[k])) if c else (lambda k: None)
    tsi = atm.get("tsi_scaling")
    args = [fused.base.ksw.handle, c.handle if c else None, ncol, nlay, P(play), P(atm["plev"]), P(atm["tlay"]),
            None, arr, len(atm["gases"]), cl("lwp"), cl("iwp"), cl("rel"), cl("rei"), int(fused.base.delta_cloud),
            P(atm["mu0"]), P(tsi) if tsi is not None else None, P(atm["sfc_alb_dir"]), P(atm["sfc_alb_dif"]),
            P(seed_up), P(seed_dn), P(seed_dir), P(seed_hr), P(grads["tlay"]), P(grads["h2o"]), P(grads["o3"]),
            P(grads["lwp"]) if c else None, P(grads["iwp"]) if c else None, P(grads["rel"]) if c else None,
            P(grads["rei"]) if c else None, P(grads["sfc_alb_dir"]), P(grads["sfc_alb_dif"])]
    fl = None
    if with_fluxes:
        fl = {k: torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev)
              for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net")}
        fl["heating_rate"] = torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
    fargs = ([P(fl[k]) for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate")] if with_fluxes
             else [None] * 5)
    if with_aerosols:
        assert fused.base.aer is not None, "solver built without aerosol tables"
        aer, keep_a = api.Gas_optics_rrtmgp._gases(atm["aerosols"], ncol, nlay, atm["play"])
        aargs = args[:2] + [fused.base.aer.handle] + args[2:15] + [aer, len(atm["aerosols"]), P(atm["rh"]),
                                                                  int(fused.base.delta_aerosol)] + args[15:]
        _abi.check(_abi.load().rrtmgp_b200_forward_adjoint_sw_aer_f32(*aargs, *fargs, api._stream()))
        return (fl, grads) if with_fluxes else grads
    if not with_fluxes:
        _abi.check(_abi.load().rrtmgp_b200_adjoint_sw_f32(*args, api._stream()))
        return grads
    _abi.check(_abi.load().rrtmgp_b200_forward_adjoint_sw_f32(*args, *fargs, api._stream()))
    return fl, grads


_SW_DIFF = ("tlay", "h2o", "o3", "lwp", "iwp", "rel", "rei", "sfc_alb_dir", "sfc_alb_dif")


class _ShortwaveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, fused, static, tlay, h2o, o3, lwp, iwp, rel, rei, alb_dir, alb_dif):
        atm = dict(static)
        atm.update(tlay=tlay, lwp=lwp, iwp=iwp, rel=rel, rei=rei, sfc_alb_dir=alb_dir, sfc_alb_dif=alb_dif)
        gases = dict(static["gases"])
        gases["h2o"], gases["o3"] = h2o, o3
        atm["gases"] = gases
        clouds = lwp is not None
        out = fused.solve_sw(atm, with_clouds=clouds)
        res = tuple(out[k].clone() for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate"))
        ctx.fused, ctx.atm, ctx.clouds = fused, atm, clouds
        ctx.save_for_backward(h2o, o3)
        return res

    @staticmethod
    def backward(ctx, g_up, g_dn, g_dir, g_net, g_hr):
        def seed(g):
            return None if g is None else g.float().contiguous()

        up, dn, dr, net, hr = map(seed, (g_up, g_dn, g_dir, g_net, g_hr))
        if net is not None:
            up = -net if up is None else up - net
            dn = net if dn is None else dn + net
        g = adjoint_sw(ctx.fused, ctx.atm, up, dn, dr, hr, with_clouds=ctx.clouds)
        h2o, o3 = ctx.saved_tensors
        out = [None, None, g["tlay"], _reduce_to(g["h2o"], h2o), _reduce_to(g["o3"], o3)]
        out += [g[k] if ctx.clouds else None for k in ("lwp", "iwp", "rel", "rei")]
        out += [g["sfc_alb_dir"], g["sfc_alb_dif"]]
        return tuple(out)


def shortwave(fused, atm: dict, with_clouds: bool = True):
    """Differentiable fused FP32 shortwave solve.  atm as for Fused_solver.solve_sw; its tlay,
    gases["h2o"], gases["o3"], lwp, iwp, rel, rei, sfc_alb_dir, sfc_alb_dif may require grad."""
    clouds = with_clouds and fused.base.csw is not None
    static = {k: v for k, v in atm.items() if k not in _SW_DIFF}
    static["gases"] = {k: v for k, v in atm["gases"].items()}
    up, dn, dr, net, hr = _ShortwaveFn.apply(
        fused, static, atm["tlay"], atm["gases"]["h2o"], atm["gases"]["o3"],
        atm["lwp"] if clouds else None, atm["iwp"] if clouds else None, atm["rel"] if clouds else None,
        atm["rei"] if clouds else None, atm["sfc_alb_dir"], atm["sfc_alb_dif"])
    return {"flux_up": up, "flux_dn": dn, "flux_dn_dir": dr, "flux_net": net, "heating_rate": hr}
