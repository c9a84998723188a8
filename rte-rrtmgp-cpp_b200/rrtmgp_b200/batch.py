"""Batched FP32 forward of many independent column grids (rrtmgp_b200_batch_* in the C ABI).

The reference runs one grid at a time, in column blocks (src_test/Radiation_solver.cu:467-615,
:683-950 called from src_test/test_rte_rrtmgp.cu); here a batch holds grids of uneven ncol and
nlay whose device arrays stay in place, and one run computes the longwave and shortwave
forwards of all of them in ONE persistent kernel launch, optionally replayed from a captured
CUDA graph.  Each grid's results equal those of Fused_solver.solve_lw / solve_sw on that grid
to FP32 rounding when the tile shape uses the same chunk length (the same per-column code,
compiled into another kernel).

Tile shapes (chunk length, columns per CTA) per (domain, 8-layer bin) come from a built-in
heuristic or from the autotuner, whose results can be cached in a JSON file keyed by the GPU
name, the domain, the k-distribution's g-point count and the bin (the reference's tuner keeps
its results in rte_rrtmgp_kernel_tuning.txt, include/tuner.h:78-182).
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import torch

from . import _abi, api

LW, SW = 0, 1
MODES = {"persistent": 0, "graph": 1, "per_grid": 2}
_P = C.c_void_p


class BatchGrid(C.Structure):
    """rrtmgp_b200_batch_grid."""
    _fields_ = [
        ("ncol", C.c_int), ("nlay", C.c_int),
        ("play", _P), ("plev", _P), ("tlay", _P), ("tlev", _P), ("tsfc", _P), ("col_dry", _P),
        ("gases", C.POINTER(_abi.GasConc)), ("ngases", C.c_int),
        ("lwp", _P), ("iwp", _P), ("rel", _P), ("rei", _P),
        ("sfc_emis", _P),
        ("lw_flux_up", _P), ("lw_flux_dn", _P), ("lw_flux_net", _P), ("lw_heating_rate", _P),
        ("mu0", _P), ("tsi_scaling", _P), ("sfc_alb_dir", _P), ("sfc_alb_dif", _P),
        ("sw_flux_up", _P), ("sw_flux_dn", _P), ("sw_flux_dn_dir", _P), ("sw_flux_net", _P),
        ("sw_heating_rate", _P),
    ]


def bins_of(nlays) -> list[int]:
    """8-layer bins (1-based, nlay in [8 bin - 7, 8 bin]) that a set of grids needs."""
    return sorted({(int(n) + 7) // 8 for n in nlays})


def cache_key(gpu: str, domain: int, ngpt: int, b: int) -> str:
    return f"{gpu}|{'lw' if domain == LW else 'sw'}|g{ngpt}|bin{b}"


def load_cache(path) -> dict:
    p = Path(path)
    if not p.exists():
        return {}
    with open(p) as f:
        d = json.load(f)
    return {k: tuple(v) for k, v in d.items()}


def save_cache(path, entries: dict):
    p = Path(path)
    old = load_cache(p)
    old.update(entries)
    p.parent.mkdir(parents=True, exist_ok=True)
    with open(p, "w") as f:
        json.dump({k: list(v) for k, v in sorted(old.items())}, f, indent=1)


def _ptr(t):
    return None if t is None else t.data_ptr()


class Batched_forward:
    """FP32 forward of a list of atmospheres (the Fused_solver input dicts, torch tensors on one
    CUDA device) through one persistent launch.

    base: a solver.Radiation_solver (k-distributions and cloud LUTs).  lw / sw select the
    domains.  Outputs are allocated here, one dict per grid and domain:
    out[i]["lw"] = {flux_up, flux_dn, flux_net (nlay+1, ncol), heating_rate (nlay, ncol)},
    out[i]["sw"] adds flux_dn_dir.  Inputs are read in place at every run, so the caller may
    overwrite them between runs (graph replays see the new values)."""

    def __init__(self, base, atms: list, with_clouds: bool = True, lw: bool = True, sw: bool = True):
        self.base = base
        self.atms = atms
        self.lw, self.sw = lw, sw
        self._keep = []
        self.out = []
        n = len(atms)
        self._grids = (BatchGrid * n)()
        cl_lw = base.clw if (with_clouds and lw) else None
        cl_sw = base.csw if (with_clouds and sw) else None
        for i, atm in enumerate(atms):
            play = atm["play"]
            assert play.dtype == torch.float32 and play.is_cuda, "batched forward takes FP32 CUDA tensors"
            nlay, ncol = play.shape
            g = self._grids[i]
            g.ncol, g.nlay = ncol, nlay
            g.play, g.plev, g.tlay = _ptr(play), _ptr(atm["plev"]), _ptr(atm["tlay"])
            g.tlev, g.tsfc = _ptr(atm.get("tlev")), _ptr(atm.get("tsfc"))
            g.col_dry = _ptr(atm.get("col_dry"))
            arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])
            self._keep += [arr, keep]
            g.gases = C.cast(arr, C.POINTER(_abi.GasConc))
            g.ngases = len(atm["gases"])
            if atm.get("lwp") is not None and (cl_lw is not None or cl_sw is not None):
                g.lwp, g.iwp, g.rel, g.rei = (_ptr(atm[k]) for k in ("lwp", "iwp", "rel", "rei"))
            o = {}
            dev = play.device
            if lw:
                o["lw"] = {k: torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev)
                           for k in ("flux_up", "flux_dn", "flux_net")}
                o["lw"]["heating_rate"] = torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
                g.sfc_emis = _ptr(atm["emis_sfc"])
                g.lw_flux_up, g.lw_flux_dn, g.lw_flux_net, g.lw_heating_rate = (
                    _ptr(o["lw"][k]) for k in ("flux_up", "flux_dn", "flux_net", "heating_rate"))
            if sw:
                o["sw"] = {k: torch.empty((nlay + 1, ncol), dtype=torch.float32, device=dev)
                           for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net")}
                o["sw"]["heating_rate"] = torch.empty((nlay, ncol), dtype=torch.float32, device=dev)
                g.mu0 = _ptr(atm["mu0"])
                g.tsi_scaling = _ptr(atm.get("tsi_scaling"))
                g.sfc_alb_dir, g.sfc_alb_dif = _ptr(atm["sfc_alb_dir"]), _ptr(atm["sfc_alb_dif"])
                g.sw_flux_up, g.sw_flux_dn, g.sw_flux_dn_dir, g.sw_flux_net, g.sw_heating_rate = (
                    _ptr(o["sw"][k]) for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net", "heating_rate"))
            self.out.append(o)
        h = _P()
        _abi.check(_abi.load().rrtmgp_b200_batch_create(
            base.klw.handle if lw else None, cl_lw.handle if cl_lw is not None else None,
            base.ksw.handle if sw else None, cl_sw.handle if cl_sw is not None else None,
            int(base.delta_cloud), C.cast(self._grids, _P), n, C.byref(h)))
        self.handle = h

    # -- running --------------------------------------------------------------------------
    def run(self, mode: str = "graph"):
        _abi.check(_abi.load().rrtmgp_b200_batch_run(self.handle, MODES[mode], api._stream()))
        return self.out

    def columns(self) -> int:
        return sum(g.ncol for g in self._grids)

    def stats(self) -> dict:
        nt, ctas, smem, lp, lg = C.c_longlong(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _abi.check(_abi.load().rrtmgp_b200_batch_stats(self.handle, C.byref(nt), C.byref(ctas), C.byref(smem),
                                                       C.byref(lp), C.byref(lg)))
        return {"tiles": nt.value, "ctas": ctas.value, "smem_bytes": smem.value,
                "launches_persistent": lp.value, "launches_per_grid": lg.value}

    # -- tile shapes ----------------------------------------------------------------------
    def domains(self):
        return [d for d, on in ((LW, self.lw), (SW, self.sw)) if on]

    def bins(self):
        return bins_of(g.nlay for g in self._grids)

    def get_plan(self, domain: int, b: int):
        cl, cols, us = C.c_int(), C.c_int(), C.c_float()
        _abi.check(_abi.load().rrtmgp_b200_batch_get_plan(self.handle, domain, b, C.byref(cl), C.byref(cols),
                                                          C.byref(us)))
        return cl.value, cols.value, us.value

    def set_plan(self, domain: int, b: int, chunk: int, columns: int, tile_us: float = 0.0):
        _abi.check(_abi.load().rrtmgp_b200_batch_set_plan(self.handle, domain, b, chunk, columns, float(tile_us)))

    def plan(self) -> dict:
        return {(d, b): self.get_plan(d, b) for d in self.domains() for b in self.bins()}

    def autotune(self, reps: int = 3, cache=None) -> dict:
        """Tile shapes for every (domain, bin) of the batch: from `cache` (a JSON file) when it
        holds them all for this GPU, else measured by rrtmgp_b200_batch_autotune (and written
        to `cache`)."""
        gpu = torch.cuda.get_device_name()
        ngpt = {LW: self.base.klw.get_ngpt(), SW: self.base.ksw.get_ngpt()}
        keys = {(d, b): cache_key(gpu, d, ngpt[d], b) for d in self.domains() for b in self.bins()}
        if cache is not None:
            c = load_cache(cache)
            if all(k in c for k in keys.values()):
                for (d, b), k in keys.items():
                    self.set_plan(d, b, *c[k])
                return self.plan()
        _abi.check(_abi.load().rrtmgp_b200_batch_autotune(self.handle, int(reps), api._stream()))
        p = self.plan()
        if cache is not None:
            save_cache(cache, {keys[db]: p[db] for db in keys})
        return p

    def close(self):
        if getattr(self, "handle", None):
            _abi.load().rrtmgp_b200_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
