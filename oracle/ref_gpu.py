"""ORACLE -- test infrastructure only.

ctypes front end of oracle/_ref/libref_rrtmgp_f64.so: the reference's own FP64 GPU classes
(rte-rrtmgp-cpp src_cuda/ + src_kernels_cuda/, built from the reference sources by
oracle/ref/Makefile) behind the C harness oracle/ref/ref_harness.cu.  Used to pin the oracle
(tests/golden/make_ref_golden.py) and, in the benchmark's reference arm, to time the
reference's GPU forward beside its CPU port.  Nothing in the product imports it.

The reference's runtime tuner (include/tuner.h) reads block shapes from
rte_rrtmgp_kernel_tuning.txt in the working directory and otherwise times many shapes on the
first call; write_tuning() writes fixed shapes first, so no tuning runs.  The minor-absorber
kernel calls __syncthreads() inside its bounds check (gas_optical_depths_minor_kernel,
gas_optics_rrtmgp_kernels.cu:386-426), so it gets a (16, 1, 1) block: every thread of a block
then shares one (column, layer) and none is out of range.  The table covers every kernel the
reference tunes (every tunings.count(...) of src_kernels_cuda/).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from rrtmgp_b200 import _abi

LIB = Path(__file__).resolve().parent / "_ref" / "libref_rrtmgp_f64.so"

REF_KERNEL_TUNING = {
    "gas_optical_depths_major_kernel": (16, 1, 8),
    "gas_optical_depths_minor_kernel_lower": (16, 1, 1),
    "gas_optical_depths_minor_kernel_upper": (16, 1, 1),
    "Planck_source_kernel": (32, 4, 1),
    "compute_tau_rayleigh_kernel": (32, 4, 1),
    "combine_abs_and_rayleigh_kernel": (32, 4, 1),
    "reorder123x321_kernel": (32, 4, 1),
    "inc_2stream_by_2stream_bybnd_kernel": (16, 4, 1),
    "lw_step_1": (32, 4, 1),
    "lw_step_2": (64, 1, 1),
    "lw_step_3": (32, 4, 1),
    "sw_source_2stream_kernel": (32, 4, 1),
    "sw_adding": (32, 4, 1),
}


def write_tuning(workdir: Path):
    """The tuner cache file, in the directory the reference library will run from."""
    with open(Path(workdir) / "rte_rrtmgp_kernel_tuning.txt", "w") as f:
        for k, (x, y, z) in REF_KERNEL_TUNING.items():
            f.write(f"{k} 1 1 1 {x} {y} {z}\n")


def load():
    lib = C.CDLL(str(LIB))
    lib.ref_last_error.restype = C.c_char_p
    return lib


def D(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def P(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def gas_array(gases):
    """GasConc array of host FP64 vmrs (scalars or (nlay, ncol) fields)."""
    arr = (_abi.GasConc * len(gases))()
    keep = []
    for i, (k, v) in enumerate(gases.items()):
        v = D(v)
        keep.append(v)
        arr[i].name = k.encode()
        arr[i].vmr = v.ctypes.data
        if v.size == 1:
            arr[i].dim1, arr[i].dim2 = 1, 1
        else:
            arr[i].dim1, arr[i].dim2 = v.shape[1], v.shape[0]
    return arr, keep


def time_forward(lib, tables: dict, atm: dict, nsteps: int = 3, ncol_block: int = 1024):
    """ref_time_forward: the reference's all-sky LW + SW forward on the GPU in blocks of
    ncol_block columns (its solve_gpu), returning (ms_lw, ms_sw, fluxes of the last step)."""
    ncol, nlay = atm["ncol"], atm["nlay"]
    tlw, k1 = _abi.kdist_tables(tables["lw"])
    tsw, k2 = _abi.kdist_tables(tables["sw"])
    clw, k3 = _abi.cloud_tables(tables["cloud_lw"])
    csw, k4 = _abi.cloud_tables(tables["cloud_sw"])
    arr, keep = gas_array(atm["gases"])
    inputs = {k: D(atm[k]) for k in ("play", "plev", "tlay", "tlev", "tsfc", "emis_sfc", "mu0", "sfc_alb_dir",
                                     "sfc_alb_dif", "lwp", "iwp", "rel", "rei")}
    out = {k: np.empty((nlay + 1, ncol)) for k in ("lw_up", "lw_dn", "sw_up", "sw_dn")}
    ms_lw, ms_sw = C.c_double(), C.c_double()
    st = lib.ref_time_forward(C.byref(tlw), C.byref(tsw), C.byref(clw), C.byref(csw), arr, len(atm["gases"]),
                              ncol, nlay, ncol_block, *(P(inputs[k]) for k in inputs), int(nsteps),
                              C.byref(ms_lw), C.byref(ms_sw), P(out["lw_up"]), P(out["lw_dn"]), P(out["sw_up"]),
                              P(out["sw_dn"]))
    if st != 0:
        raise RuntimeError(lib.ref_last_error().decode())
    return ms_lw.value, ms_sw.value, out
