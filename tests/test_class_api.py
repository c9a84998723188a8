"""The C++ class API (include/cpp: Gas_optics_rrtmgp_gpu, Cloud_optics_gpu, Rte_lw_gpu,
Rte_sw_gpu, Fluxes_broadband_gpu, ...) driven the way the reference's
Radiation_solver::solve_gpu drives it (tests/cpp/class_api_driver.cpp), in both Float
precisions, against the FP64 oracle.

CPU tests: the headers compile for Float = double and float, and both driver libraries load
and report their Float size.  GPU tests: LW/SW all-sky and clear-sky parity (Float = double:
the staged FP64 tolerances; Float = float: the staged FP32 tolerances) and the missing-gas
constructor error.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from rrtmgp_b200 import _abi
from rrtmgp_b200 import synthetic as S

REPO = Path(__file__).resolve().parents[1]
CPP = REPO / "tests" / "cpp"
FLUX_RTOL = {8: 1e-8, 4: 2e-4}
FLUX_FLOOR = {8: 1e-4, 4: 1e-2}


def _driver(fbytes):
    lib_path = CPP / "_build" / ("libclass_api_f64.so" if fbytes == 8 else "libclass_api_f32.so")
    if not lib_path.exists():
        subprocess.run(["make", "-s", "-C", str(CPP)], check=True)
    _abi.load()
    return C.CDLL(str(lib_path))


def test_headers_compile_both_precisions(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text("".join(f'#include "{h}"\n' for h in ("Gas_optics_rrtmgp.h", "Cloud_optics.h", "Aerosol_optics.h",
                                                          "Rte_lw.h", "Rte_sw.h", "Fluxes.h")) +
                   "int main() { return 0; }\n")
    for flag in ([], ["-DRTE_USE_SP"]):
        subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", *flag,
                        f"-I{REPO / 'include' / 'cpp'}", "-I/usr/local/cuda/include", str(src)], check=True)


@pytest.mark.parametrize("fbytes", [8, 4])
def test_driver_loads(fbytes):
    lib = _driver(fbytes)
    assert lib.class_api_float_bytes() == fbytes


def _gas_args(atm):
    names = list(atm["gases"].keys())
    arrs = [np.ascontiguousarray(np.asarray(atm["gases"][n], np.float64)) for n in names]
    dims = []
    for a in arrs:
        dims += [1, 1] if a.size == 1 else [a.shape[1], a.shape[0]]
    keep = [n.encode() for n in names]
    name_arr = (C.c_char_p * len(names))(*keep)
    vmr_arr = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    dim_arr = (C.c_int * len(dims))(*dims)
    return (len(names), name_arr, vmr_arr, dim_arr), (keep, arrs)


def _cmp(name, got, ref, fbytes):
    floor = FLUX_FLOOR[fbytes] * np.max(np.abs(ref))
    err = np.max(np.abs(got - ref) / (np.abs(ref) + floor))
    assert err <= FLUX_RTOL[fbytes], f"{name}: max rel err {err:.3e} (Float of {fbytes} bytes)"


def _ptrs(d, keys):
    return [d[k].ctypes.data_as(C.c_void_p) for k in keys]


def _run_lw(fbytes, tables, atm, clouds):
    lib = _driver(fbytes)
    kt, keep_t = _abi.kdist_tables(tables["lw"])
    ct, keep_c = _abi.cloud_tables(tables["cloud_lw"])
    gargs, keep_g = _gas_args(atm)
    nlay, ncol = atm["play"].shape
    inp = {k: np.ascontiguousarray(np.asarray(atm[k], np.float64))
           for k in ("play", "plev", "tlay", "tlev", "tsfc", "emis_sfc", "lwp", "iwp", "rel", "rei")}
    out = {k: np.zeros((nlay + 1, ncol)) for k in ("flux_up", "flux_dn", "flux_net")}
    err = C.create_string_buffer(512)
    st = lib.class_api_forward_lw(C.byref(kt), C.byref(ct) if clouds else None, ncol, nlay,
                                  *_ptrs(inp, ("play", "plev", "tlay", "tlev", "tsfc", "emis_sfc")), *gargs,
                                  *_ptrs(inp, ("lwp", "iwp", "rel", "rei")), 1,
                                  *_ptrs(out, ("flux_up", "flux_dn", "flux_net")), err, 512)
    assert st == 0, err.value.decode()
    return out


def _run_sw(fbytes, tables, atm, clouds):
    lib = _driver(fbytes)
    kt, keep_t = _abi.kdist_tables(tables["sw"])
    ct, keep_c = _abi.cloud_tables(tables["cloud_sw"])
    gargs, keep_g = _gas_args(atm)
    nlay, ncol = atm["play"].shape
    inp = {k: np.ascontiguousarray(np.asarray(atm[k], np.float64))
           for k in ("play", "plev", "tlay", "mu0", "tsi_scaling", "sfc_alb_dir", "sfc_alb_dif",
                     "lwp", "iwp", "rel", "rei")}
    keys = ("flux_up", "flux_dn", "flux_dn_dir", "flux_net")
    out = {k: np.zeros((nlay + 1, ncol)) for k in keys}
    err = C.create_string_buffer(512)
    st = lib.class_api_forward_sw(C.byref(kt), C.byref(ct) if clouds else None, ncol, nlay,
                                  *_ptrs(inp, ("play", "plev", "tlay", "mu0", "tsi_scaling", "sfc_alb_dir",
                                               "sfc_alb_dif")), *gargs,
                                  *_ptrs(inp, ("lwp", "iwp", "rel", "rei")), *_ptrs(out, keys), err, 512)
    assert st == 0, err.value.decode()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("fbytes", [8, 4])
@pytest.mark.parametrize("clouds", [False, True])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_class_api_lw(oracle_mod, tables, gpu, fbytes, clouds, top_at_1):
    atm = S.make_atmosphere(41, 50, seed=11, clouds=clouds, top_at_1=top_at_1)
    ref = oracle_mod.forward_lw(oracle_mod.GasOptics(tables["lw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_lw"]) if clouds else None, atm)
    got = _run_lw(fbytes, tables, atm, clouds)
    for k in ("flux_up", "flux_dn", "flux_net"):
        _cmp(f"lw {k}", got[k], ref[k], fbytes)


@pytest.mark.gpu
@pytest.mark.parametrize("fbytes", [8, 4])
@pytest.mark.parametrize("clouds", [False, True])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_class_api_sw(oracle_mod, tables, gpu, fbytes, clouds, top_at_1):
    atm = S.make_atmosphere(41, 50, seed=12, clouds=clouds, top_at_1=top_at_1)
    atm["tsi_scaling"] = np.linspace(0.95, 1.05, 41)
    ref = oracle_mod.forward_sw(oracle_mod.GasOptics(tables["sw"], S.ATM_GASES),
                                oracle_mod.CloudOptics(tables["cloud_sw"]) if clouds else None, atm)
    got = _run_sw(fbytes, tables, atm, clouds)
    for k in ("flux_up", "flux_dn", "flux_dn_dir"):
        _cmp(f"sw {k}", got[k], ref[k], fbytes)


@pytest.mark.gpu
def test_class_api_missing_key_species_throws(tables, gpu):
    lib = _driver(8)
    kt, keep = _abi.kdist_tables(tables["lw"])
    err = C.create_string_buffer(512)
    assert lib.class_api_missing_gas_throws(C.byref(kt), err, 512) == 0
    assert "missing" in err.value.decode().lower()


@pytest.mark.gpu
@pytest.mark.parametrize("fbytes", [8, 4])
def test_aerosol_optics_class(oracle_mod, gpu, fbytes):
    """Aerosol_optics_gpu::aerosol_optics (Aerosol_concs with profile and field species)
    against the oracle."""
    lib = _driver(fbytes)
    tab = S.make_aerosol_luts()
    ta, keep_t = _abi.aerosol_tables(tab)
    ncol, nlay = 6, 15
    atm = S.make_atmosphere(ncol, nlay, seed=61, clouds=False)
    aer, rh = S.make_aerosols(atm["play"], seed=62)
    aer["aermr03"] = aer["aermr03"][:, 0].copy()   # a profile, broadcast over the columns
    ref = oracle_mod.aerosol_optics(tab, aer, rh, atm["plev"])
    args, keep = _gas_args({"gases": {k: (v[:, None] if v.ndim == 1 else v) for k, v in aer.items()}})
    out = {k: np.empty((14, nlay, ncol)) for k in ("tau", "ssa", "g")}
    err = C.create_string_buffer(256)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rh_c = np.ascontiguousarray(rh)
    pl_c = np.ascontiguousarray(atm["plev"])
    st = lib.class_api_aerosol_optics(C.byref(ta), ncol, nlay, P(rh_c), P(pl_c), *args, P(out["tau"]),
                                      P(out["ssa"]), P(out["g"]), err, 256)
    assert st == 0, err.value.decode()
    feps = np.finfo(np.float32 if fbytes == 4 else np.float64).eps
    rtol = 1e-12 if fbytes == 8 else 2e-6
    m = {"tau": np.ones(out["tau"].shape, bool), "ssa": ref["tau"] > 2 * feps, "g": ref["tau"] * ref["ssa"] > 2 * feps}
    for k in out:
        np.testing.assert_allclose(out[k][m[k]], ref[k][m[k]], rtol=rtol, atol=1e-30, err_msg=k)
