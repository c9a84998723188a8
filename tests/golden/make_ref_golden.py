"""Generates the golden fixtures that pin the oracle to the reference implementation.

Runs the reference's own FP64 GPU classes (rte-rrtmgp-cpp src_cuda/ + src_kernels_cuda/,
compiled by oracle/ref/Makefile into oracle/_ref/libref_rrtmgp_f64.so) on small seeded
synthetic cases and stores inputs and outputs as compressed npz files:

    python tests/golden/make_ref_golden.py OUTDIR [--only dense]   # on a machine with a GPU

--only dense writes only the gas-optics fixtures of the dense tables (make_kdist(dense=True):
every halocarbon, up to 13 minor intervals in a band and 11 over one g-point).

The reference's runtime tuner would otherwise time many block shapes on first use; its cache
file (rte_rrtmgp_kernel_tuning.txt, read from the working directory, include/tuner.h:50-61)
is written first with fixed block shapes, so no tuning runs.  The minor-absorber kernel calls
__syncthreads() inside its bounds check (gas_optical_depths_minor_kernel,
gas_optics_rrtmgp_kernels.cu:386-426), so it gets a (16, 1, 1) block: every thread of a block
then shares one (column, layer) and none is out of range.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(REPO), str(REPO / "rte-rrtmgp-cpp_b200")]

from rrtmgp_b200 import _abi, synthetic as S  # noqa: E402

LIB = REPO / "oracle" / "_ref" / "libref_rrtmgp_f64.so"

from oracle.ref_gpu import REF_KERNEL_TUNING as TUNING, D, P, gas_array  # noqa: E402

NCOL, NLAY = 5, 10


def addto_inputs():
    """Random 2str gas (224 g-points) and cloud (14 bands) properties of the add_to case."""
    rng = np.random.default_rng(104)
    gas = {"tau": rng.uniform(0, 2, (224, NLAY, NCOL)), "ssa": rng.uniform(0, 1, (224, NLAY, NCOL)),
           "g": rng.uniform(0, 0.9, (224, NLAY, NCOL))}
    cld = {"tau": rng.uniform(0, 5, (14, NLAY, NCOL)), "ssa": rng.uniform(0.5, 1, (14, NLAY, NCOL)),
           "g": rng.uniform(0.7, 0.9, (14, NLAY, NCOL))}
    return gas, cld


def flux_inputs():
    """Random g-point fluxes (224 g-points) of the reduction case."""
    rng = np.random.default_rng(105)
    return tuple(rng.uniform(0, 20, (224, NLAY + 1, NCOL)) for _ in range(3))


def aerosol_inputs(atm):
    """Mixing ratios aermr01 .. aermr11 and relative humidity of the aerosol case."""
    aer, rh = S.make_aerosols(atm["play"], seed=108)
    aer["aermr05"] = np.array([3e-9])
    return aer, rh


def dense_gas_cases(lib, chk, outdir: Path):
    """Gas optics of the dense tables (LW top-at-1 and bottom-at-1, SW top-at-1) on a
    trace-gas atmosphere."""
    lw, sw = S.make_kdist("lw", dense=True), S.make_kdist("sw", dense=True)
    tlw, k1 = _abi.kdist_tables(lw)
    tsw, k2 = _abi.kdist_tables(sw)
    for name, top in (("gas_lw_dense_top1", True), ("gas_lw_dense_bot1", False)):
        atm = S.make_atmosphere(NCOL, NLAY, seed=111, clouds=False, top_at_1=top, trace_gases=True)
        arr, keep = gas_array(atm["gases"])
        o = {k: np.empty((256, NLAY, NCOL)) for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec")}
        o["sfc_src"] = np.empty((256, NCOL))
        o["sfc_src_jac"] = np.empty((256, NCOL))
        chk(lib.ref_gas_optics_lw(C.byref(tlw), arr, len(atm["gases"]), NCOL, NLAY, P(D(atm["play"])),
                                  P(D(atm["plev"])), P(D(atm["tlay"])), P(D(atm["tsfc"])), P(D(atm["tlev"])), None,
                                  P(o["tau"]), P(o["lay_src"]), P(o["lev_src_inc"]), P(o["lev_src_dec"]),
                                  P(o["sfc_src"]), P(o["sfc_src_jac"])))
        np.savez_compressed(outdir / f"{name}.npz", seed=111, top_at_1=top, **o)
    atm = S.make_atmosphere(NCOL, NLAY, seed=112, clouds=False, top_at_1=True, trace_gases=True)
    arr, keep = gas_array(atm["gases"])
    o = {k: np.empty((224, NLAY, NCOL)) for k in ("tau", "ssa", "g")}
    o["toa_src"] = np.empty((224, NCOL))
    chk(lib.ref_gas_optics_sw(C.byref(tsw), arr, len(atm["gases"]), NCOL, NLAY, P(D(atm["play"])),
                              P(D(atm["plev"])), P(D(atm["tlay"])), None, P(o["tau"]), P(o["ssa"]), P(o["g"]),
                              P(o["toa_src"])))
    np.savez_compressed(outdir / "gas_sw_dense_top1.npz", seed=112, top_at_1=True, **o)


def main(outdir: Path, only: str = ""):
    outdir = outdir.resolve()
    outdir.mkdir(parents=True, exist_ok=True)
    workdir = outdir / "_tuner_cwd"
    workdir.mkdir(exist_ok=True)
    with open(workdir / "rte_rrtmgp_kernel_tuning.txt", "w") as f:
        for k, (x, y, z) in TUNING.items():
            f.write(f"{k} 1 1 1 {x} {y} {z}\n")
    os.chdir(workdir)
    lib = C.CDLL(str(LIB))
    lib.ref_last_error.restype = C.c_char_p

    def chk(st):
        if st != 0:
            raise RuntimeError(lib.ref_last_error().decode())

    if only == "dense":
        dense_gas_cases(lib, chk, outdir)
        print("golden fixtures written to", outdir)
        return
    lw, sw = S.make_kdist("lw"), S.make_kdist("sw")
    clw, csw = S.make_cloud_luts("lw"), S.make_cloud_luts("sw")
    tlw, k1 = _abi.kdist_tables(lw)
    tsw, k2 = _abi.kdist_tables(sw)

    # Gas optics, both orientations (col_dry computed by the reference when not given).
    for name, top, with_cd in (("gas_lw_top1", True, False), ("gas_lw_bot1", False, True)):
        atm = S.make_atmosphere(NCOL, NLAY, seed=101, clouds=False, top_at_1=top)
        cd = D(S.col_dry_from(atm["gases"]["h2o"], atm["plev"])) if with_cd else None
        arr, keep = gas_array(atm["gases"])
        o = {k: np.empty((256, NLAY, NCOL)) for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec")}
        o["sfc_src"] = np.empty((256, NCOL))
        o["sfc_src_jac"] = np.empty((256, NCOL))
        chk(lib.ref_gas_optics_lw(C.byref(tlw), arr, len(atm["gases"]), NCOL, NLAY, P(D(atm["play"])),
                                  P(D(atm["plev"])), P(D(atm["tlay"])), P(D(atm["tsfc"])), P(D(atm["tlev"])), P(cd),
                                  P(o["tau"]), P(o["lay_src"]), P(o["lev_src_inc"]), P(o["lev_src_dec"]),
                                  P(o["sfc_src"]), P(o["sfc_src_jac"])))
        np.savez_compressed(outdir / f"{name}.npz", seed=101, top_at_1=top, with_col_dry=with_cd, **o)
    for name, top in (("gas_sw_top1", True), ("gas_sw_bot1", False)):
        atm = S.make_atmosphere(NCOL, NLAY, seed=102, clouds=False, top_at_1=top)
        arr, keep = gas_array(atm["gases"])
        o = {k: np.empty((224, NLAY, NCOL)) for k in ("tau", "ssa", "g")}
        o["toa_src"] = np.empty((224, NCOL))
        chk(lib.ref_gas_optics_sw(C.byref(tsw), arr, len(atm["gases"]), NCOL, NLAY, P(D(atm["play"])),
                                  P(D(atm["plev"])), P(D(atm["tlay"])), None, P(o["tau"]), P(o["ssa"]), P(o["g"]),
                                  P(o["toa_src"])))
        np.savez_compressed(outdir / f"{name}.npz", seed=102, top_at_1=top, **o)

    # Cloud optics.
    atm = S.make_atmosphere(NCOL, NLAY, seed=103, clouds=True)
    for name, tab, two, delta in (("cloud_lw_1scl", clw, 0, 0), ("cloud_sw_2str", csw, 1, 0),
                                  ("cloud_sw_2str_delta", csw, 1, 1)):
        ct, k3 = _abi.cloud_tables(tab)
        nb = ct.nband
        o = {"tau": np.empty((nb, NLAY, NCOL))}
        if two:
            o["ssa"] = np.empty_like(o["tau"])
            o["g"] = np.empty_like(o["tau"])
        chk(lib.ref_cloud_optics(C.byref(ct), NCOL, NLAY, P(D(atm["lwp"])), P(D(atm["iwp"])), P(D(atm["rel"])),
                                 P(D(atm["rei"])), two, delta, P(o["tau"]), P(o.get("ssa")), P(o.get("g"))))
        np.savez_compressed(outdir / f"{name}.npz", seed=103, **o)

    # add_to by band.
    bl = D(sw["bnd_limits_gpt"]).astype(np.int32)
    gas, cld = addto_inputs()
    o = {k: gas[k].copy() for k in gas}
    chk(lib.ref_add_to_2str_bybnd(NCOL, NLAY, 14, bl.ctypes.data_as(C.POINTER(C.c_int)), P(o["tau"]), P(o["ssa"]),
                                  P(o["g"]), P(D(cld["tau"])), P(D(cld["ssa"])), P(D(cld["g"]))))
    np.savez_compressed(outdir / "add_to_2str_bybnd.npz", **o)
    rng = np.random.default_rng(106)

    # Longwave solver on the reference's own gas optics of the top_at_1 case.
    g = np.load(outdir / "gas_lw_top1.npz")
    bll = D(lw["bnd_limits_gpt"]).astype(np.int32)
    emis = rng.uniform(0.85, 1.0, (NCOL, 16))
    up, dn = np.empty((256, NLAY + 1, NCOL)), np.empty((256, NLAY + 1, NCOL))
    chk(lib.ref_rte_lw(NCOL, NLAY, 16, bll.ctypes.data_as(C.POINTER(C.c_int)), 1, P(D(g["tau"])),
                       P(D(g["lay_src"])), P(D(g["lev_src_inc"])), P(D(g["lev_src_dec"])), P(D(g["sfc_src"])),
                       P(D(emis)), P(up), P(dn)))
    np.savez_compressed(outdir / "rte_lw_top1.npz", emis=emis, flux_up=up, flux_dn=dn)

    # Shortwave solver on the reference's gas optics; albedo uniform across bands (the
    # reference CUDA kernel uses the first g-point's direct albedo for every g-point).
    for name, gname, top in (("rte_sw_top1", "gas_sw_top1", 1), ("rte_sw_bot1", "gas_sw_bot1", 0)):
        g = np.load(outdir / f"{gname}.npz")
        alb = np.repeat(rng.uniform(0.05, 0.3, NCOL)[:, None], 14, axis=1)
        albf = np.repeat(rng.uniform(0.05, 0.3, NCOL)[:, None], 14, axis=1)
        mu0 = rng.uniform(0.1, 1.0, NCOL)
        up, dn, dr = (np.empty((224, NLAY + 1, NCOL)) for _ in range(3))
        chk(lib.ref_rte_sw(NCOL, NLAY, 14, bl.ctypes.data_as(C.POINTER(C.c_int)), top, P(D(g["tau"])),
                           P(D(g["ssa"])), P(D(g["g"])), P(D(mu0)), P(D(g["toa_src"])), P(D(alb)), P(D(albf)),
                           P(up), P(dn), P(dr)))
        np.savez_compressed(outdir / f"{name}.npz", alb_dir=alb, alb_dif=albf, mu0=mu0, flux_up=up, flux_dn=dn,
                            flux_dir=dr)

    # Aerosol optics (shortwave) on seeded synthetic tables and mixing ratios, bottom-up
    # column order, one species given as a scalar.
    aer_tab, keep_aer = _abi.aerosol_tables(S.make_aerosol_luts())
    atm = S.make_atmosphere(NCOL, NLAY, seed=107, clouds=False, top_at_1=False)
    aer, rh = aerosol_inputs(atm)
    arr, keep = gas_array(aer)
    o = {k: np.empty((14, NLAY, NCOL)) for k in ("tau", "ssa", "g")}
    chk(lib.ref_aerosol_optics(C.byref(aer_tab), arr, len(aer), NCOL, NLAY, P(D(rh)), P(D(atm["plev"])),
                               P(o["tau"]), P(o["ssa"]), P(o["g"])))
    np.savez_compressed(outdir / "aerosol_sw.npz", **o)

    # Flux reductions.
    gu, gd, gr = flux_inputs()
    bb = {k: np.empty((NLAY + 1, NCOL)) for k in ("flux_up", "flux_dn", "flux_dn_dir", "flux_net")}
    by = {k: np.empty((14, NLAY + 1, NCOL)) for k in ("bnd_flux_up", "bnd_flux_dn", "bnd_flux_net")}
    chk(lib.ref_fluxes(NCOL, NLAY + 1, 14, bl.ctypes.data_as(C.POINTER(C.c_int)), P(gu), P(gd), P(gr),
                       P(bb["flux_up"]), P(bb["flux_dn"]), P(bb["flux_dn_dir"]), P(bb["flux_net"]),
                       P(by["bnd_flux_up"]), P(by["bnd_flux_dn"]), P(by["bnd_flux_net"])))
    np.savez_compressed(outdir / "fluxes.npz", **bb, **by)
    print("golden fixtures written to", outdir)


if __name__ == "__main__":
    if len(sys.argv) not in (2, 4) or (len(sys.argv) == 4 and sys.argv[2:] != ["--only", "dense"]):
        sys.exit("usage: python tests/golden/make_ref_golden.py OUTPUT_DIR [--only dense]")
    main(Path(sys.argv[1]), sys.argv[3] if len(sys.argv) == 4 else "")
