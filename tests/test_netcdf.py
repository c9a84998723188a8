"""Coefficient-table I/O: the netCDF-4 (HDF5) reader of rrtmgp_b200.netcdf.

The reference ships one netCDF-4 file, data/aerosol_optics.nc (read by its
load_and_init_aerosol_optics, src_test/Radiation_solver.cu:366-401); where the reference
checkout is present it is decoded here and run through the aerosol optics of the oracle.  The
k-distribution and cloud files (rrtmgp-data) are not in the checkout, so their loaders are
exercised through the same reader only when such files are supplied (RRTMGP_DATA_DIR); the
table loaders themselves are checked on netCDF classic and 64-bit-offset files that scipy's
writer makes from the synthetic tables (the same variable names and layouts).
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


def _write_classic(path, tables, version):
    """Write a table dict (netCDF variable names, C order, strings as lists) as a netCDF
    classic (version 1) or 64-bit-offset (version 2) file with scipy's writer."""
    from scipy.io import netcdf_file
    f = netcdf_file(str(path), "w", version=version)
    for k, v in tables.items():
        if k == "kind" or v is None:
            continue
        if isinstance(v, list):
            width = max([1] + [len(x) for x in v])
            a = np.zeros((len(v), width), "S1")
            for i, x in enumerate(v):
                a[i, :len(x)] = [bytes([c]) for c in x.encode()]
            f.createDimension(f"{k}_n", a.shape[0])
            f.createDimension(f"{k}_len", width)
            f.createVariable(k, "c", (f"{k}_n", f"{k}_len"))[:] = a
        elif np.ndim(v) == 0:
            f.createVariable(k, "d", ())[...] = float(v)
        else:
            a = np.asarray(v)
            dims = []
            for i, n in enumerate(a.shape):
                f.createDimension(f"{k}_{i}", n)
                dims.append(f"{k}_{i}")
            f.createVariable(k, "i" if a.dtype.kind == "i" else "d", tuple(dims))[:] = a
    f.close()


def _same_tables(got, want):
    for k, v in want.items():
        if k == "kind":
            continue
        if v is None:
            assert got[k] is None, k
        elif isinstance(v, list):
            assert got[k] == v, k
        else:
            g = np.asarray(got[k])
            assert g.shape == np.shape(v), (k, g.shape, np.shape(v))
            assert np.array_equal(g, np.asarray(v)), k


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("kind", ["lw", "sw"])
def test_gas_optics_tables_round_trip_classic(tmp_path, kind, version):
    """load_gas_optics on a classic / 64-bit-offset file written by scipy from the synthetic
    k-distribution returns the same tables, strings and scalars included."""
    t = S.make_kdist(kind)
    p = tmp_path / f"gas_{kind}.nc"
    _write_classic(p, t, version)
    got = N.load_gas_optics(p)
    assert got["kind"] == kind
    _same_tables(got, t)
    assert got["kmajor"].dtype == np.float64 and got["bnd_limits_gpt"].dtype == np.int32


@pytest.mark.parametrize("kind", ["lw", "sw"])
def test_cloud_and_aerosol_tables_round_trip_classic(tmp_path, kind):
    c = S.make_cloud_luts(kind)
    p = tmp_path / "cloud.nc"
    _write_classic(p, c, 2)
    got = N.load_cloud_optics(p, kind)
    assert got["kind"] == kind
    for k in ("lut_extliq", "lut_ssaliq", "lut_asyliq", "lut_extice", "lut_ssaice", "lut_asyice",
              "bnd_limits_wavenumber"):
        assert np.array_equal(got[k], c[k]), k
    for k in ("radliq_lwr", "radliq_upr", "radice_lwr", "radice_upr", "radliq_fac", "radice_fac"):
        assert float(got[k]) == float(np.asarray(c[k]).reshape(-1)[0]), k
    a = S.make_aerosol_luts()
    pa = tmp_path / "aerosol.nc"
    _write_classic(pa, {k: a[k] for k in N._AEROSOL_VARS}, 1)
    ga = N.load_aerosol_optics(pa)
    for k in N._AEROSOL_VARS:
        assert np.array_equal(ga[k], a[k]), k


def test_classic_reader_types_records_and_errors(tmp_path):
    """Every classic type, a record variable interleaved with another one, and the errors."""
    from scipy.io import netcdf_file
    p = tmp_path / "types.nc"
    f = netcdf_file(str(p), "w", version=2)
    f.createDimension("t", None)
    f.createDimension("x", 3)
    vals = {"b": ("b", np.array([-1, 2, 3], np.int8)), "h": ("h", np.array([-300, 2, 7], np.int16)),
            "i": ("i", np.array([-70000, 1, 2], np.int32)), "f": ("f", np.array([1.5, -2.25, 3e10], np.float32)),
            "d": ("d", np.array([1e-300, 2.0, -3.5]))}
    for k, (code, a) in vals.items():
        f.createVariable(k, code, ("x",))[:] = a
    r1 = f.createVariable("r1", "d", ("t", "x"))
    r2 = f.createVariable("r2", "h", ("t",))
    for r in range(4):
        r1[r] = np.arange(3) + 10.0 * r
        r2[r] = r - 2
    f.close()
    c = N.ClassicFile(p)
    assert sorted(c.variables()) == sorted(list(vals) + ["r1", "r2"])
    for k, (_, a) in vals.items():
        got = c.read(k)
        assert got.dtype == a.dtype.newbyteorder("=") and np.array_equal(got, a), k
    assert np.array_equal(c.read("r1"), np.arange(3)[None, :] + 10.0 * np.arange(4)[:, None])
    assert np.array_equal(c.read("r2"), np.arange(4) - 2)
    assert N.read_netcdf(p).keys() == set(c.variables())
    with pytest.raises(N.NetcdfError, match="no variable"):
        c.read("zz")
    bad = tmp_path / "v5.nc"
    bad.write_bytes(b"CDF\x05" + bytes(60))
    with pytest.raises(N.NetcdfError, match="version 5"):
        N.read_netcdf(bad)
    short = tmp_path / "short.nc"
    short.write_bytes(p.read_bytes()[:40])
    with pytest.raises(N.NetcdfError):
        N.read_netcdf(short)


@pytest.mark.parametrize("style", [0, 2])
def test_hdf5_symbol_table_v1_headers_and_chunked_filters(tmp_path, style):
    """The reader's superblock-0 / v1-header / symbol-table path and every storage layout it
    decodes, on a file written by tests/h5_writer.py: compact, contiguous, unallocated (read as
    zeros), chunked with partial edge chunks under a one- and a two-level chunk B-tree, filter
    pipelines of version 1 (shuffle + deflate) and 2 (deflate + fletcher32, one chunk stored with
    deflate skipped), big- and little-endian numbers, NC_CHAR strings and a nested group.  Style
    2 writes the same datasets under superblock 2 with version-2 headers and link messages."""
    from h5_writer import H5Writer, Dataset, SHUFFLE, DEFLATE, FLETCHER32
    rng = np.random.default_rng(4)
    k3 = rng.standard_normal((5, 7, 9)).astype(np.float32)
    i2 = rng.integers(-3000, 3000, (11, 6)).astype(np.int16)
    names = np.array([[bytes([c]) for c in f"{s:<4}".encode()] for s in ("h2o", "co2", "o3")], "S1")
    members = {
        "kmajor": Dataset(k3, "chunked", chunks=(2, 4, 9), filters=[SHUFFLE, DEFLATE], leaf=3),
        "counts": Dataset(i2, "chunked", chunks=(4, 6), filters=[DEFLATE, FLETCHER32], pipeline_version=2,
                          skip={(4, 0): 1}),
        "press_ref": Dataset(np.linspace(1.0, 1e5, 13), "contiguous"),
        "big_endian": Dataset(np.arange(6, dtype=">i4").reshape(2, 3), "contiguous"),
        "key_species": Dataset(np.arange(8, dtype=np.int32), "compact"),
        "compact_big": Dataset(np.arange(100, dtype=np.float64), "compact"),   # header over 255 bytes
        "tsi_default": Dataset(np.array(1360.9), "contiguous"),
        "gas_names": Dataset(names, "contiguous"),
        "never_written": Dataset(np.zeros((3, 2)), "unallocated"),
        "sub": {"inner": Dataset(np.array([1.5, 2.5], np.float64), "chunked", chunks=(1,), filters=[DEFLATE])},
    }
    p = tmp_path / f"v{style}.nc"
    H5Writer(style).write(p, members)
    f = N.H5File(p)
    assert f.variables() == sorted(["kmajor", "counts", "press_ref", "big_endian", "key_species", "compact_big",
                                    "tsi_default", "gas_names", "never_written", "sub/inner"])
    assert np.array_equal(f.read("compact_big"), np.arange(100.0))
    assert np.array_equal(f.read("kmajor"), k3) and f.read("kmajor").dtype == np.float32
    assert np.array_equal(f.read("counts"), i2)
    assert np.array_equal(f.read("press_ref"), members["press_ref"].data)
    got = f.read("big_endian")
    assert got.dtype == np.dtype("=i4") and np.array_equal(got, np.arange(6).reshape(2, 3))
    assert np.array_equal(f.read("key_species"), np.arange(8))
    assert float(f.read("tsi_default")) == 1360.9
    assert N._strings(f.read("gas_names")) == ["h2o", "co2", "o3"]
    assert np.array_equal(f.read("never_written"), np.zeros((3, 2)))
    assert np.array_equal(f.read("sub/inner"), [1.5, 2.5])
    assert set(N.read_netcdf(p)) == set(f.variables())


def test_hdf5_aerosol_tables_round_trip(tmp_path):
    """load_aerosol_optics on an HDF5 file of the synthetic aerosol tables (chunked and
    deflated, as netCDF-4 writes compressed variables)."""
    from h5_writer import H5Writer, Dataset, SHUFFLE, DEFLATE
    a = S.make_aerosol_luts()
    members = {}
    for k in N._AEROSOL_VARS:
        v = np.asarray(a[k])
        members[k] = Dataset(v, "chunked", chunks=tuple(max(1, n // 2) for n in v.shape), filters=[SHUFFLE, DEFLATE])
    p = tmp_path / "aerosol_h5.nc"
    H5Writer().write(p, members)
    got = N.load_aerosol_optics(p)
    for k in N._AEROSOL_VARS:
        assert np.array_equal(got[k], a[k]), k
