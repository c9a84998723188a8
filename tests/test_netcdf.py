"""Coefficient-table I/O: the netCDF-4 (HDF5) reader of rrtmgp_b200.netcdf.

The reference ships one netCDF-4 file, data/aerosol_optics.nc (read by its
load_and_init_aerosol_optics, src_test/Radiation_solver.cu:366-401); where the reference
checkout is present it is decoded here and run through the aerosol optics of the oracle.  The
k-distribution and cloud files (rrtmgp-data) are not in the checkout, so their loaders are
exercised through the same reader only when such files are supplied (RRTMGP_DATA_DIR).
"""
import os
from pathlib import Path

import numpy as np
import pytest

from rrtmgp_b200 import netcdf as N
from rrtmgp_b200 import synthetic as S

AEROSOL_FILE = Path("/root/reference/data/aerosol_optics.nc")
DATA_DIR = os.environ.get("RRTMGP_DATA_DIR")


def test_strings_from_char_arrays():
    a = np.array([[b"h", b"2", b"o", b" "], [b"o", b"3", b"\0", b"\0"]], dtype="S1")
    assert N._strings(a) == ["h2o", "o3"]
    assert N._strings(np.array([b"co2  ", b"n2o\0\0"])) == ["co2", "n2o"]


def test_rejects_a_file_that_is_not_hdf5(tmp_path):
    p = tmp_path / "x.nc"
    p.write_bytes(b"CDF\x01" + bytes(600))      # a classic netCDF header is not HDF5
    with pytest.raises(N.NetcdfError, match="not an HDF5"):
        N.H5File(p)


@pytest.mark.skipif(not AEROSOL_FILE.exists(), reason="reference checkout not present")
def test_reads_the_reference_aerosol_tables(oracle_mod):
    f = N.H5File(AEROSOL_FILE)
    names = f.variables()
    for k in N._AEROSOL_VARS:
        assert k in names
    with pytest.raises(N.NetcdfError, match="no variable"):
        f.read("kmajor")
    t = N.load_aerosol_optics(AEROSOL_FILE)
    rh = t["relative_humidity2"]
    nhum = rh.size
    nphobic, nband = t["mass_ext_sw_hydrophobic"].shape
    nphilic = t["mass_ext_sw_hydrophilic"].shape[0]
    assert nband == 14 and nphobic >= 11 and nphilic >= 5
    assert t["mass_ext_sw_hydrophilic"].shape == (nphilic, nhum, nband)
    assert np.all(np.diff(rh) > 0) and 0.0 < rh[0] and rh[-1] <= 1.0
    for k in ("ssa_sw_hydrophobic", "ssa_sw_hydrophilic"):
        assert np.all((t[k] >= 0.0) & (t[k] <= 1.0))
    for k in ("asymmetry_sw_hydrophobic", "asymmetry_sw_hydrophilic"):
        assert np.all(np.abs(t[k]) <= 1.0)
    assert np.all(t["mass_ext_sw_hydrophobic"] > 0.0) and np.all(t["mass_ext_sw_hydrophilic"] >= 0.0)
    # char variables decode to species codes of two letters
    assert all(len(c) == 2 for c in N._strings(f.read("code_hydrophobic")))

    # the tables drive the oracle's aerosol optics like the synthetic ones
    atm = S.make_atmosphere(16, 30, seed=3, clouds=False)
    aer, rhf = S.make_aerosols(atm["play"], seed=5)
    out = oracle_mod.aerosol_optics(t, aer, rhf, atm["plev"])
    assert out["tau"].shape == (nband, 30, 16)
    assert np.all(np.isfinite(out["tau"])) and np.all(out["tau"] > 0.0)
    assert np.all((out["ssa"] >= 0.0) & (out["ssa"] <= 1.0))
    assert np.all(np.abs(out["g"]) <= 1.0)


@pytest.mark.skipif(not DATA_DIR, reason="RRTMGP coefficient files not supplied")
def test_loads_supplied_rrtmgp_files():
    d = Path(DATA_DIR)
    for name, kind in (("rrtmgp-gas-lw-g256.nc", "lw"), ("rrtmgp-gas-sw-g224.nc", "sw")):
        if (d / name).exists():
            t = N.load_gas_optics(d / name)
            assert t["kind"] == kind and t["kmajor"].ndim == 4 and "h2o" in t["gas_names"]
    for name in ("rrtmgp-clouds-lw.nc", "rrtmgp-clouds-sw.nc"):
        if (d / name).exists():
            c = N.load_cloud_optics(d / name)
            assert c["lut_extice"].ndim == 3
