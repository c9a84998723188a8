"""ctypes view of the C ABI declared in include/rrtmgp_b200.h."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "librrtmgp_b200.so"

OK, ERR_ARG, ERR_RANGE, ERR_MISSING_GAS, ERR_CUDA, ERR_ALLOC, ERR_UNSUPPORTED, ERR_WORKSPACE = range(8)

c_int_p = C.POINTER(C.c_int)
c_double_p = C.POINTER(C.c_double)
c_char_pp = C.POINTER(C.c_char_p)


class KdistTables(C.Structure):
    _fields_ = [
        ("ngas", C.c_int), ("nband", C.c_int), ("ngpt", C.c_int), ("ntemp", C.c_int),
        ("npres", C.c_int), ("neta", C.c_int), ("nminor_absorber", C.c_int),
        ("nint_lower", C.c_int), ("nint_upper", C.c_int),
        ("ncontrib_lower", C.c_int), ("ncontrib_upper", C.c_int), ("nplanck_temp", C.c_int),
        ("gas_names", c_char_pp), ("key_species", c_int_p), ("band_lims_gpt", c_int_p),
        ("band_lims_wvn", c_double_p), ("press_ref", c_double_p), ("press_ref_trop", C.c_double),
        ("temp_ref", c_double_p), ("temp_ref_p", C.c_double), ("temp_ref_t", C.c_double),
        ("vmr_ref", c_double_p), ("kmajor", c_double_p),
        ("kminor_lower", c_double_p), ("kminor_upper", c_double_p),
        ("gas_minor", c_char_pp), ("identifier_minor", c_char_pp),
        ("minor_gases_lower", c_char_pp), ("minor_gases_upper", c_char_pp),
        ("minor_limits_gpt_lower", c_int_p), ("minor_limits_gpt_upper", c_int_p),
        ("minor_scales_with_density_lower", c_int_p), ("minor_scales_with_density_upper", c_int_p),
        ("scaling_gas_lower", c_char_pp), ("scaling_gas_upper", c_char_pp),
        ("scale_by_complement_lower", c_int_p), ("scale_by_complement_upper", c_int_p),
        ("kminor_start_lower", c_int_p), ("kminor_start_upper", c_int_p),
        ("totplnk", c_double_p), ("planck_frac", c_double_p),
        ("solar_source_quiet", c_double_p), ("solar_source_facular", c_double_p),
        ("solar_source_sunspot", c_double_p),
        ("tsi_default", C.c_double), ("mg_default", C.c_double), ("sb_default", C.c_double),
        ("rayl_lower", c_double_p), ("rayl_upper", c_double_p),
    ]


class CloudTables(C.Structure):
    _fields_ = [
        ("nband", C.c_int), ("nsize_liq", C.c_int), ("nsize_ice", C.c_int), ("nrghice", C.c_int),
        ("band_lims_wvn", c_double_p),
        ("radliq_lwr", C.c_double), ("radliq_upr", C.c_double), ("radliq_fac", C.c_double),
        ("radice_lwr", C.c_double), ("radice_upr", C.c_double), ("radice_fac", C.c_double),
        ("lut_extliq", c_double_p), ("lut_ssaliq", c_double_p), ("lut_asyliq", c_double_p),
        ("lut_extice", c_double_p), ("lut_ssaice", c_double_p), ("lut_asyice", c_double_p),
    ]


class AerosolTables(C.Structure):
    _fields_ = [
        ("nband", C.c_int), ("nhum", C.c_int), ("nphilic", C.c_int), ("nphobic", C.c_int),
        ("rh_upper", c_double_p), ("mext_phobic", c_double_p), ("ssa_phobic", c_double_p),
        ("g_phobic", c_double_p), ("mext_philic", c_double_p), ("ssa_philic", c_double_p),
        ("g_philic", c_double_p),
    ]


class GasConc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("vmr", C.c_void_p), ("dim1", C.c_int), ("dim2", C.c_int)]


class KdistInfo(C.Structure):
    _fields_ = [
        ("ngas", C.c_int), ("nflav", C.c_int), ("nband", C.c_int), ("ngpt", C.c_int),
        ("ntemp", C.c_int), ("npres", C.c_int), ("neta", C.c_int), ("nplanck_temp", C.c_int),
        ("nminor_lower", C.c_int), ("nminor_upper", C.c_int),
        ("is_longwave", C.c_int), ("has_rayleigh", C.c_int),
        ("press_ref_min", C.c_double), ("press_ref_max", C.c_double),
        ("temp_ref_min", C.c_double), ("temp_ref_max", C.c_double), ("tsi", C.c_double),
    ]


class _Keep:
    """Holds the numpy buffers and string arrays a ctypes structure points into."""

    def __init__(self):
        self.refs = []

    def f64(self, a):
        if a is None:
            return None
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        self.refs.append(arr)
        return arr.ctypes.data_as(c_double_p)

    def i32(self, a):
        if a is None:
            return None
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
        self.refs.append(arr)
        return arr.ctypes.data_as(c_int_p)

    def strs(self, lst):
        bufs = [C.c_char_p(s.encode()) for s in lst]
        arr = (C.c_char_p * max(len(bufs), 1))(*bufs)
        self.refs.append((bufs, arr))
        return C.cast(arr, c_char_pp)


def kdist_tables(d: dict):
    """ctypes KdistTables for a k-distribution dict in netCDF layout; returns (struct, keep)."""
    k = _Keep()
    t = KdistTables()
    ngas = len(d["gas_names"])
    km = np.asarray(d["kmajor"])
    t.ngas = ngas
    t.nband = len(d["bnd_limits_gpt"])
    t.ngpt = km.shape[3]
    t.ntemp = len(d["temp_ref"])
    t.npres = len(d["press_ref"])
    t.neta = km.shape[2]
    t.nminor_absorber = len(d["identifier_minor"])
    t.nint_lower = len(d["minor_gases_lower"])
    t.nint_upper = len(d["minor_gases_upper"])
    t.ncontrib_lower = np.asarray(d["kminor_lower"]).shape[2]
    t.ncontrib_upper = np.asarray(d["kminor_upper"]).shape[2]
    t.nplanck_temp = np.asarray(d["totplnk"]).shape[1] if d.get("totplnk") is not None else 0
    t.gas_names = k.strs(d["gas_names"])
    t.key_species = k.i32(d["key_species"])
    t.band_lims_gpt = k.i32(d["bnd_limits_gpt"])
    t.band_lims_wvn = k.f64(d["bnd_limits_wavenumber"])
    t.press_ref = k.f64(d["press_ref"])
    t.press_ref_trop = float(d["press_ref_trop"])
    t.temp_ref = k.f64(d["temp_ref"])
    t.temp_ref_p = float(d["absorption_coefficient_ref_P"])
    t.temp_ref_t = float(d["absorption_coefficient_ref_T"])
    t.vmr_ref = k.f64(d["vmr_ref"])
    t.kmajor = k.f64(km)
    t.kminor_lower = k.f64(d["kminor_lower"])
    t.kminor_upper = k.f64(d["kminor_upper"])
    t.gas_minor = k.strs(d["gas_minor"])
    t.identifier_minor = k.strs(d["identifier_minor"])
    t.minor_gases_lower = k.strs(d["minor_gases_lower"])
    t.minor_gases_upper = k.strs(d["minor_gases_upper"])
    t.minor_limits_gpt_lower = k.i32(d["minor_limits_gpt_lower"])
    t.minor_limits_gpt_upper = k.i32(d["minor_limits_gpt_upper"])
    t.minor_scales_with_density_lower = k.i32(d["minor_scales_with_density_lower"])
    t.minor_scales_with_density_upper = k.i32(d["minor_scales_with_density_upper"])
    t.scaling_gas_lower = k.strs(d["scaling_gas_lower"])
    t.scaling_gas_upper = k.strs(d["scaling_gas_upper"])
    t.scale_by_complement_lower = k.i32(d["scale_by_complement_lower"])
    t.scale_by_complement_upper = k.i32(d["scale_by_complement_upper"])
    t.kminor_start_lower = k.i32(d["kminor_start_lower"])
    t.kminor_start_upper = k.i32(d["kminor_start_upper"])
    t.totplnk = k.f64(d.get("totplnk"))
    t.planck_frac = k.f64(d.get("plank_fraction"))
    t.solar_source_quiet = k.f64(d.get("solar_source_quiet"))
    t.solar_source_facular = k.f64(d.get("solar_source_facular"))
    t.solar_source_sunspot = k.f64(d.get("solar_source_sunspot"))
    t.tsi_default = float(d.get("tsi_default", 0.0))
    t.mg_default = float(d.get("mg_default", 0.0))
    t.sb_default = float(d.get("sb_default", 0.0))
    t.rayl_lower = k.f64(d.get("rayl_lower"))
    t.rayl_upper = k.f64(d.get("rayl_upper"))
    return t, k


def aerosol_tables(d: dict):
    """ctypes AerosolTables for an aerosol LUT dict in netCDF layout (the variables that
    load_and_init_aerosol_optics reads); returns (struct, keep)."""
    k = _Keep()
    t = AerosolTables()
    ph = np.asarray(d["mass_ext_sw_hydrophobic"])
    pl = np.asarray(d["mass_ext_sw_hydrophilic"])
    t.nphobic, t.nband = ph.shape
    t.nphilic, t.nhum = pl.shape[0], pl.shape[1]
    t.rh_upper = k.f64(d["relative_humidity2"])
    t.mext_phobic = k.f64(ph)
    t.ssa_phobic = k.f64(d["ssa_sw_hydrophobic"])
    t.g_phobic = k.f64(d["asymmetry_sw_hydrophobic"])
    t.mext_philic = k.f64(pl)
    t.ssa_philic = k.f64(d["ssa_sw_hydrophilic"])
    t.g_philic = k.f64(d["asymmetry_sw_hydrophilic"])
    return t, k


def cloud_tables(d: dict):
    k = _Keep()
    t = CloudTables()
    ext_l = np.asarray(d["lut_extliq"])
    ext_i = np.asarray(d["lut_extice"])
    t.nband = ext_l.shape[0]
    t.nsize_liq = ext_l.shape[1]
    t.nsize_ice = ext_i.shape[2]
    t.nrghice = ext_i.shape[0]
    t.band_lims_wvn = k.f64(d["bnd_limits_wavenumber"])
    for name in ("radliq_lwr", "radliq_upr", "radliq_fac", "radice_lwr", "radice_upr", "radice_fac"):
        setattr(t, name, float(d[name]))
    for name in ("lut_extliq", "lut_ssaliq", "lut_asyliq", "lut_extice", "lut_ssaice", "lut_asyice"):
        setattr(t, name, k.f64(d[name]))
    return t, k


def string_array(names):
    k = _Keep()
    return k.strs(names), k


_P = C.c_void_p
_I = C.c_int
_SZ = C.c_size_t

# name -> (restype, argtypes); FP entry points are listed once with a placeholder for _f32/_f64.
_SIGS = {
    "rrtmgp_b200_last_error": (C.c_char_p, []),
    "rrtmgp_b200_abi_version": (_I, []),
    "rrtmgp_b200_kdist_create": (_I, [C.POINTER(KdistTables), c_char_pp, _I, C.POINTER(_P)]),
    "rrtmgp_b200_kdist_destroy": (None, [_P]),
    "rrtmgp_b200_kdist_get_info": (_I, [_P, C.POINTER(KdistInfo)]),
    "rrtmgp_b200_kdist_gas_name": (_I, [_P, _I, C.c_char_p, _I]),
    "rrtmgp_b200_kdist_bands": (_P, [_P]),
    "rrtmgp_b200_kdist_set_solar_variability": (_I, [_P, C.c_double, C.c_double]),
    "rrtmgp_b200_kdist_solar_source": (_I, [_P, c_double_p]),
    "rrtmgp_b200_bands_create": (_I, [_I, c_int_p, C.POINTER(_P)]),
    "rrtmgp_b200_bands_destroy": (None, [_P]),
    "rrtmgp_b200_bands_get": (_I, [_P, c_int_p, c_int_p]),
    "rrtmgp_b200_cloud_create": (_I, [C.POINTER(CloudTables), C.POINTER(_P)]),
    "rrtmgp_b200_cloud_destroy": (None, [_P]),
    "rrtmgp_b200_rte_sw_workspace_bytes": (_SZ, [_I, _I, _I, _I]),
    "rrtmgp_b200_device_wait_timeouts": (_I, [C.POINTER(C.c_uint)]),
    "rrtmgp_b200_rte_sw_static_scratch_f32": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rrtmgp_b200_forward_lw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                        _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "rrtmgp_b200_forward_sw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                        _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "rrtmgp_b200_forward_sw_aer_f32": (_I, [_P, _P, _P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                            _P, _P, _P, _P, _I, C.POINTER(GasConc), _I, _P, _I,
                                            _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "rrtmgp_b200_fp32_fma_probe": (_I, [_I, _I, _P, _P]),
    "rrtmgp_b200_aerosol_create": (_I, [C.POINTER(AerosolTables), C.POINTER(_P)]),
    "rrtmgp_b200_aerosol_destroy": (None, [_P]),
    "rrtmgp_b200_forward_adjoint_lw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                                _P, _P, _P, _P, _P, _P, _P, _P,
                                                _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "rrtmgp_b200_forward_adjoint_sw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                                _P, _P, _P, _P, _I, _P, _P, _P, _P,
                                                _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                                _P, _P, _P, _P, _P, _P]),
    "rrtmgp_b200_forward_adjoint_sw_aer_f32": (_I, [_P, _P, _P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                                    _P, _P, _P, _P, _I, C.POINTER(GasConc), _I, _P, _I,
                                                    _P, _P, _P, _P,
                                                    _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                                    _P, _P, _P, _P, _P, _P]),
    "rrtmgp_b200_rte_sw_abs_f32": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rrtmgp_b200_heating_rate_from_layer_abs_f32": (_I, [_I, _I, _I, _P, _P, _P, _P]),
    "rrtmgp_b200_batch_create": (_I, [_P, _P, _P, _P, _I, _P, _I, C.POINTER(_P)]),
    "rrtmgp_b200_batch_destroy": (_I, [_P]),
    "rrtmgp_b200_batch_run": (_I, [_P, _I, _P]),
    "rrtmgp_b200_batch_autotune": (_I, [_P, _I, _P]),
    "rrtmgp_b200_batch_get_plan": (_I, [_P, _I, _I, c_int_p, c_int_p, C.POINTER(C.c_float)]),
    "rrtmgp_b200_batch_set_plan": (_I, [_P, _I, _I, _I, _I, C.c_float]),
    "rrtmgp_b200_batch_stats": (_I, [_P, C.POINTER(C.c_longlong), c_int_p, c_int_p, c_int_p, c_int_p]),
    "rrtmgp_b200_adjoint_sw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                        _P, _P, _P, _P, _I, _P, _P, _P, _P,
                                        _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rrtmgp_b200_adjoint_lw_f32": (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                                        _P, _P, _P, _P, _P, _P, _P, _P,
                                        _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
}
SW_STATIC_SCRATCH_MAX_ELEMS = 1048576
_FP_SIGS = {
    "get_col_dry": [_I, _I, _P, _P, _P, _P],
    "gas_optics_lw": [_P, _I, _I, _P, _P, _P, _P, _P, _P, C.POINTER(GasConc), _I,
                      _P, _P, _P, _P, _P, _P, _P],
    "gas_optics_sw": [_P, _I, _I, _P, _P, _P, _P, C.POINTER(GasConc), _I, _P, _P, _P, _P, _P],
    "check_range": [_P, _I, _I, _P, _P, _P, _P, _P, _P, _P],
    "cloud_optics_1scl": [_P, _I, _I, _P, _P, _P, _P, _P, _P],
    "cloud_optics_2str": [_P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P],
    "delta_scale_2str": [_I, _I, _I, _P, _P, _P, _P],
    "add_to_1scl": [_P, _I, _I, _P, _P, _I, _P],
    "add_to_2str": [_P, _I, _I, _P, _P, _P, _P, _P, _P, _I, _P],
    "rte_lw": [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P],
    "rte_lw_jac": [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P],
    "rte_sw": [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P],
    "fluxes_broadband": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P],
    "fluxes_byband": [_P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P],
    "heating_rate": [_I, _I, _P, _P, _P, _P, _P],
    "heating_rate_lw_layers": [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "heating_rate_sw_layers": [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "aerosol_optics": [_P, _I, _I, C.POINTER(GasConc), _I, _P, _P, _P, _P, _P, _P],
}


def declared_symbols():
    """Every function name the C header declares (used by the ABI export test)."""
    names = list(_SIGS)
    for base in _FP_SIGS:
        names += [f"rrtmgp_b200_{base}_f32", f"rrtmgp_b200_{base}_f64"]
    return names


_lib = None


def load(path: Path = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not Path(path).exists():
        raise RuntimeError(f"rrtmgp_b200 CUDA library missing at {path}; run rte-rrtmgp-cpp_b200/build.py")
    lib = C.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    for base, args in _FP_SIGS.items():
        for sfx in ("_f32", "_f64"):
            f = getattr(lib, f"rrtmgp_b200_{base}{sfx}")
            f.restype = _I
            f.argtypes = args
    _lib = lib
    return lib


class RrtmgpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"rrtmgp_b200 status {status}: {msg}")
        self.status = status


def check(status):
    if status != OK:
        raise RrtmgpError(status, load().rrtmgp_b200_last_error().decode())
    return status
