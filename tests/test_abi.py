"""CPU tests of the C ABI boundary: the library loads without a GPU and exports every
function include/rrtmgp_b200.h declares; the Python table marshalling is consistent."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from rrtmgp_b200 import _abi, synthetic as S

HEADER = Path(__file__).resolve().parent.parent / "include" / "rrtmgp_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rrtmgp_b200_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_match_binding():
    assert sorted(_abi.declared_symbols()) == declared_functions()


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_abi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.rrtmgp_b200_abi_version() == 1


def test_binding_signatures_load():
    lib = _abi.load()
    assert lib.rrtmgp_b200_last_error() is not None


def test_workspace_query_needs_no_gpu():
    lib = _abi.load()
    # on-chip solver up to 256 layers (FP32) / 128 (FP64): no workspace
    assert lib.rrtmgp_b200_rte_sw_workspace_bytes(10, 20, 30, 0) == 0
    assert lib.rrtmgp_b200_rte_sw_workspace_bytes(10, 256, 30, 0) == 0
    assert lib.rrtmgp_b200_rte_sw_workspace_bytes(10, 129, 30, 1) == 4 * 10 * 129 * 30 * 8
    assert lib.rrtmgp_b200_rte_sw_workspace_bytes(10, 257, 30, 0) == 4 * 10 * 257 * 30 * 4


def test_null_arguments_are_rejected_without_gpu():
    lib = _abi.load()
    st = lib.rrtmgp_b200_kdist_create(None, None, 0, None)
    assert st == _abi.ERR_ARG
    assert b"null" in lib.rrtmgp_b200_last_error()


def test_every_entry_point_rejects_null_arguments():
    """Every compute and handle entry point validates its arguments before any CUDA call:
    with null handles and pointers and zero sizes each returns RRTMGP_B200_ERR_ARG and
    leaves a message naming itself, on a machine with or without a GPU."""
    lib = _abi.load()
    no_status = {"rrtmgp_b200_abi_version", "rrtmgp_b200_last_error",
                 "rrtmgp_b200_rte_sw_workspace_bytes", "rrtmgp_b200_kdist_bands"}
    checked = 0
    for name in sorted(_abi.declared_symbols()):
        if name in no_status or name.endswith("_destroy"):
            continue
        f = getattr(lib, name)
        args = [0 if a in (ctypes.c_int, ctypes.c_long, ctypes.c_ulong)
                else 0.0 if a in (ctypes.c_float, ctypes.c_double) else None
                for a in f.argtypes]
        assert f(*args) == _abi.ERR_ARG, name
        msg = lib.rrtmgp_b200_last_error().decode()
        stem = name[len("rrtmgp_b200_"):].removesuffix("_f32").removesuffix("_f64")
        assert msg.split(":")[0] in stem, (name, msg)
        checked += 1
    assert checked >= 50
    for name in ("kdist", "cloud", "aerosol", "bands"):
        getattr(lib, f"rrtmgp_b200_{name}_destroy")(None)      # destroying NULL is a no-op
    assert lib.rrtmgp_b200_batch_destroy(None) in (0, _abi.ERR_ARG)


@pytest.mark.parametrize("case", ["gap", "overlap", "short", "reversed"])
def test_kdist_create_rejects_band_limits_with_gaps(tables, case):
    """Band limits must cover g-points 1..ngpt in order (the kernels walk the g-points band
    after band); kdist_create refuses other layouts before any device allocation."""
    import ctypes as C
    d = dict(tables["lw"])
    lims = np.array(d["bnd_limits_gpt"], copy=True)
    if case == "gap":
        lims[3, 0] += 1
    elif case == "overlap":
        lims[3, 0] -= 1
    elif case == "short":
        lims[-1, 1] -= 1
    else:
        lims[[2, 3]] = lims[[3, 2]]
    d["bnd_limits_gpt"] = lims
    lib = _abi.load()
    t, keep = _abi.kdist_tables(d)
    names, keep2 = _abi.string_array(list(S.ATM_GASES))
    h = C.c_void_p()
    assert lib.rrtmgp_b200_kdist_create(C.byref(t), names, len(S.ATM_GASES), C.byref(h)) == _abi.ERR_ARG
    assert b"band limits" in lib.rrtmgp_b200_last_error()
    assert not h.value


def test_table_struct_dimensions(tables):
    t, keep = _abi.kdist_tables(tables["lw"])
    assert (t.nband, t.ngpt, t.ntemp, t.npres, t.neta) == (16, 256, 14, 59, 9)
    assert t.nplanck_temp == 196 and t.ncontrib_lower == tables["lw"]["kminor_lower"].shape[2]
    ts, keep2 = _abi.kdist_tables(tables["sw"])
    assert ts.nplanck_temp == 0 and bool(ts.rayl_lower) and not bool(ts.totplnk)
    c, keep3 = _abi.cloud_tables(tables["cloud_sw"])
    assert (c.nband, c.nsize_liq, c.nsize_ice, c.nrghice) == (14, 20, 18, 3)


def test_synthetic_atmosphere_layout():
    atm = S.make_atmosphere(7, 9, seed=1)
    assert atm["play"].shape == (9, 7) and atm["plev"].shape == (10, 7)
    assert np.all(np.diff(atm["plev"][:, 0]) > 0)  # top_at_1: pressure increases with index
    assert atm["plev"][0, 0] >= S.PRESS_REF_MIN
    flip = S.make_atmosphere(7, 9, seed=1, top_at_1=False)
    assert np.all(np.diff(flip["plev"][:, 0]) < 0)


def test_gas_concentrations_are_validated_before_any_pointer_is_taken():
    """Gas_concs entries reach the kernels as raw pointers read in the call's precision, so a
    host tensor, another dtype or an unknown shape is refused on the host (no GPU needed)."""
    import torch
    from rrtmgp_b200 import api
    nlay, ncol = 6, 5
    play = torch.ones((nlay, ncol), dtype=torch.float32)
    with pytest.raises(ValueError, match="dtype"):
        api.Gas_optics_rrtmgp._gases({"h2o": torch.ones((nlay, ncol), dtype=torch.float64)}, ncol, nlay, play)
    with pytest.raises(ValueError, match="CUDA"):
        api.Gas_optics_rrtmgp._gases({"h2o": torch.ones((nlay, ncol), dtype=torch.float32)}, ncol, nlay, play)
    with pytest.raises(ValueError, match="shape"):
        api.Gas_optics_rrtmgp._gases({"o3": torch.ones((ncol, nlay), dtype=torch.float32)}, ncol, nlay, play)
    with pytest.raises(ValueError, match="torch tensor"):
        api.Gas_optics_rrtmgp._gases({"co2": np.ones(1, np.float32)}, ncol, nlay, play)
