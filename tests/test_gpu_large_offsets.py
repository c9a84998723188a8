"""Staged FP32 kernels on a grid whose (column, level, g-point) offsets pass 2^31.

The packed gas optics, the chunked shortwave solver (with and without its absorbed-flux
output) and the heating-rate kernels use 32-bit offsets when every offset of a call fits in
31 bits and 64-bit offsets otherwise.  Every other test runs the 32-bit instances; here a
1024-column atmosphere is tiled 586 times along the columns (600,064 columns of 16 layers,
offsets up to 2.46e9), so the same kernels run their 64-bit instances, and every tiled block,
the last one included, must reproduce the 1024-column call.  About 63 GB of device memory at the peak; skipped when less is free.
"""

import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

NC, NLAY, REPS = 1024, 16, 586


def _tile(atm_small):
    """The device atmosphere repeated REPS times along its column axis."""
    out = {}
    for k, v in atm_small.items():
        if k == "gases":
            out[k] = {g: (x.repeat(1, REPS) if x.dim() == 2 and x.shape[1] == NC else x) for g, x in v.items()}
        elif not hasattr(v, "dim"):
            out[k] = v
        elif v.dim() == 1 and v.shape[0] == NC:
            out[k] = v.repeat(REPS)
        elif v.dim() == 2 and v.shape[1] == NC:
            out[k] = v.repeat(1, REPS)
        elif v.dim() == 2 and v.shape[0] == NC:
            out[k] = v.repeat(REPS, 1)
        else:
            out[k] = v
    return out


def _blocks(big, small, what):
    """Compares the column blocks 0, 1, REPS // 2 and REPS - 1 of big (..., REPS * NC) with small."""
    s = small.double().cpu().numpy()
    floor = 1e-6 * max(float(np.abs(s).max()), 1e-30)
    for b in (0, 1, REPS // 2, REPS - 1):
        got = big[..., b * NC:(b + 1) * NC].double().cpu().numpy()
        err = np.max(np.abs(got - s) / (np.abs(s) + floor))
        assert err <= 1e-6, f"{what}: column block {b} differs from the 1024-column call by {err:.3e}"


def _need_memory(gpu, gib):
    import torch
    torch.cuda.synchronize(gpu)
    torch.cuda.empty_cache()
    free = torch.cuda.mem_get_info(gpu)[0]
    if free < gib * 2**30:
        pytest.skip(f"needs {gib} GiB of free device memory, {free / 2**30:.0f} GiB free")


@pytest.fixture(scope="module")
def small_atm(gpu):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    return atm_to_device(S.make_atmosphere(NC, NLAY, seed=61, clouds=False), torch.float32, gpu)


@pytest.mark.gpu
def test_longwave_offsets_past_2_31(tables, gpu, small_atm):
    import torch
    from rrtmgp_b200 import _abi, api
    assert NC * REPS * NLAY * 256 >= 2**31
    _need_memory(gpu, 72)
    kd = api.Gas_optics_rrtmgp(tables["lw"], S.ATM_GASES)
    lib = _abi.load()
    top = bool(small_atm["play"][0, 0] < small_atm["play"][-1, 0])

    def run(a, ncol):
        go = kd.gas_optics_lw(a["play"], a["plev"], a["tlay"], a["tsfc"], a["gases"], a["tlev"])
        up, dn = api.Rte_lw.rte_lw(kd.bands, go["tau"], top, go, a["emis_sfc"])
        hr = torch.empty((NLAY, ncol), dtype=torch.float32, device=gpu)
        _abi.check(lib.rrtmgp_b200_heating_rate_lw_layers_f32(
            ncol, NLAY, go["tau"].shape[0], int(top), api._ptr(go["tau"]), api._ptr(go["lay_src"]),
            api._ptr(go["lev_src_inc"]), api._ptr(go["lev_src_dec"]), api._ptr(up), api._ptr(dn),
            api._ptr(a["plev"]), api._ptr(hr), api._stream()))
        return go, up, dn, hr

    ref = run(small_atm, NC)
    big = run(_tile(small_atm), NC * REPS)
    torch.cuda.synchronize(gpu)
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec"):
        _blocks(big[0][k], ref[0][k], "gas_optics_lw " + k)
    _blocks(big[1], ref[1], "rte_lw flux_up")
    _blocks(big[2], ref[2], "rte_lw flux_dn")
    _blocks(big[3], ref[3], "heating_rate_lw_layers")
    del big
    torch.cuda.empty_cache()


@pytest.mark.gpu
def test_shortwave_offsets_past_2_31(tables, gpu, small_atm):
    import torch
    from rrtmgp_b200 import _abi, api
    assert NC * REPS * NLAY * 224 >= 2**31
    _need_memory(gpu, 72)
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    lib = _abi.load()
    top = bool(small_atm["play"][0, 0] < small_atm["play"][-1, 0])

    def run(a, ncol):
        go = kd.gas_optics_sw(a["play"], a["plev"], a["tlay"], a["gases"])
        up, dn, dr = api.Rte_sw.rte_sw(kd.bands, go["tau"], go["ssa"], go["g"], top, a["mu0"], go["toa_src"],
                                       a["sfc_alb_dir"], a["sfc_alb_dif"])
        hr = torch.empty((NLAY, ncol), dtype=torch.float32, device=gpu)
        _abi.check(lib.rrtmgp_b200_heating_rate_sw_layers_f32(
            ncol, NLAY, go["tau"].shape[0], int(top), api._ptr(go["tau"]), api._ptr(go["ssa"]),
            api._ptr(go["g"]), api._ptr(a["mu0"]), api._ptr(up), api._ptr(dn), api._ptr(dr),
            api._ptr(a["plev"]), api._ptr(hr), api._stream()))
        # the solver that also writes each layer's absorbed flux (its fluxes, within FP32 rounding
        # of rte_sw's, overwrite those), and the heating rate summed from it
        layer_abs = torch.empty_like(go["tau"])
        hr2 = torch.empty((NLAY, ncol), dtype=torch.float32, device=gpu)
        _abi.check(lib.rrtmgp_b200_rte_sw_abs_f32(
            kd.bands.handle, ncol, NLAY, int(top), api._ptr(go["tau"]), api._ptr(go["ssa"]), api._ptr(go["g"]),
            api._ptr(a["mu0"]), api._ptr(go["toa_src"]), api._ptr(a["sfc_alb_dir"]), api._ptr(a["sfc_alb_dif"]),
            None, api._ptr(up), api._ptr(dn), api._ptr(dr), api._ptr(layer_abs), api._stream()))
        _abi.check(lib.rrtmgp_b200_heating_rate_from_layer_abs_f32(
            ncol, NLAY, go["tau"].shape[0], api._ptr(layer_abs), api._ptr(a["plev"]), api._ptr(hr2), api._stream()))
        return go, up, dn, dr, hr, layer_abs, hr2

    ref = run(small_atm, NC)
    big = run(_tile(small_atm), NC * REPS)
    torch.cuda.synchronize(gpu)
    for k in ("tau", "ssa"):
        _blocks(big[0][k], ref[0][k], "gas_optics_sw " + k)
    _blocks(big[1], ref[1], "rte_sw flux_up")
    _blocks(big[2], ref[2], "rte_sw flux_dn")
    _blocks(big[3], ref[3], "rte_sw flux_dir")
    _blocks(big[4], ref[4], "heating_rate_sw_layers")
    _blocks(big[5], ref[5], "rte_sw_abs layer_abs")
    _blocks(big[6], ref[6], "heating_rate_from_layer_abs")
    del big
    torch.cuda.empty_cache()
