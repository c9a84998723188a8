"""Dense minor-absorber layouts on the GPU.

The dense tables (synthetic.make_kdist(..., dense=True)) list every gas of the public LW g256
file, halocarbons included, with 13 minor intervals in one band, seven intervals over the same
g-points in two bands and up to 11 intervals over one g-point, and the atmospheres carry all
of those gases (make_atmosphere(..., trace_gases=True)).  Every product kernel runs on them
and is compared with the FP64 oracle with the bounds of the other GPU tests: the fused
forwards (5e-3 W/m2, 0.01 K/day), the staged gas optics (FP32 2e-4, FP64 1e-10 relative), both
adjoints (central differences, 3e-3 of max|FD|) and the batched persistent kernel.
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

from test_gpu_adjoint import _check, _fd, _fd_bands, _get, _informative, _seeds, _sw_seeds
from test_gpu_stages import N, T, cmp, dtypes

pytestmark = pytest.mark.gpu
GASES = S.ATM_GASES_DENSE
HR_TOL = 0.01
FLUX_TOL = 5e-3


@pytest.fixture(scope="module")
def dense():
    return {"lw": S.make_kdist("lw", dense=True), "sw": S.make_kdist("sw", dense=True),
            "cloud_lw": S.make_cloud_luts("lw"), "cloud_sw": S.make_cloud_luts("sw")}


def _solvers(dense):
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver
    base = Radiation_solver(dense["lw"], dense["sw"], dense["cloud_lw"], dense["cloud_sw"], GASES)
    return base, Fused_solver(base)


def _oracle(oracle_mod, dense, atm, clouds=True):
    glw, gsw = oracle_mod.GasOptics(dense["lw"], GASES), oracle_mod.GasOptics(dense["sw"], GASES)
    clw = oracle_mod.CloudOptics(dense["cloud_lw"]) if clouds else None
    csw = oracle_mod.CloudOptics(dense["cloud_sw"]) if clouds else None
    return oracle_mod.forward_lw(glw, clw, atm), oracle_mod.forward_sw(gsw, csw, atm)


def _check_fluxes(got, ref, what):
    for k in ref:
        if k not in got:
            continue
        e = np.max(np.abs(got[k].double().cpu().numpy() - ref[k]))
        tol = HR_TOL if k == "heating_rate" else FLUX_TOL
        assert e < tol, f"{what} {k}: {e:.3e}"


def test_dense_kdist_is_accepted_by_every_fused_path(dense, gpu):
    from rrtmgp_b200 import api
    for kind in ("lw", "sw"):
        kd = api.Gas_optics_rrtmgp(dense[kind], GASES)
        assert kd.info.nminor_lower >= 60 and kd.info.nminor_upper >= 60
        assert kd.info.ngas == len(S.GAS_NAMES_DENSE)


@pytest.mark.parametrize("nlay", [60, 128])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_fused_forward_dense_matches_oracle(oracle_mod, dense, gpu, nlay, top_at_1):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(dense)
    atm = S.make_atmosphere(33, nlay, seed=90 + nlay, clouds=True, top_at_1=top_at_1, trace_gases=True)
    rlw, rsw = _oracle(oracle_mod, dense, atm)
    d = atm_to_device(atm, torch.float32, gpu)
    lw, sw = fused.solve_lw(d), fused.solve_sw(d)
    torch.cuda.synchronize()
    _check_fluxes(lw, rlw, f"dense lw nlay={nlay} top_at_1={top_at_1}")
    _check_fluxes(sw, rsw, f"dense sw nlay={nlay} top_at_1={top_at_1}")


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("top_at_1", [True, False])
def test_staged_gas_optics_dense_matches_oracle(oracle_mod, dense, gpu, prec, top_at_1):
    from rrtmgp_b200 import api
    dt = dtypes()[prec]
    atm = S.make_atmosphere(37, 23, seed=93, clouds=False, top_at_1=top_at_1, trace_gases=True)
    g = {k: T(v.reshape(1) if v.size == 1 else v, dt, gpu) for k, v in atm["gases"].items()}
    ref = oracle_mod.GasOptics(dense["lw"], GASES).gas_optics_lw(
        atm["play"], atm["plev"], atm["tlay"], atm["tsfc"], atm["gases"], atm["tlev"])
    got = api.Gas_optics_rrtmgp(dense["lw"], GASES).gas_optics_lw(
        T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu), T(atm["tsfc"], dt, gpu), g,
        T(atm["tlev"], dt, gpu))
    for k in ("tau", "lay_src", "lev_src_inc", "lev_src_dec", "sfc_src", "sfc_src_jac"):
        cmp("dense lw " + k, N(got[k]), ref[k], prec)
    ref = oracle_mod.GasOptics(dense["sw"], GASES).gas_optics_sw(atm["play"], atm["plev"], atm["tlay"], atm["gases"])
    got = api.Gas_optics_rrtmgp(dense["sw"], GASES).gas_optics_sw(
        T(atm["play"], dt, gpu), T(atm["plev"], dt, gpu), T(atm["tlay"], dt, gpu), g)
    for k in ("tau", "ssa", "toa_src"):
        cmp("dense sw " + k, N(got[k]), ref[k], prec)


def test_lw_adjoint_dense_matches_fd(oracle_mod, dense, gpu):
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw
    from rrtmgp_b200.solver import atm_to_device
    rng = np.random.default_rng(13)
    ncol, nlay = 2, 20
    atm = S.make_atmosphere(ncol, nlay, seed=95, clouds=True, trace_gases=True)
    kd, cl = oracle_mod.GasOptics(dense["lw"], GASES), oracle_mod.CloudOptics(dense["cloud_lw"])
    fwd = lambda a: oracle_mod.forward_lw(kd, cl, a)  # noqa: E731
    seeds = _seeds(nlay, ncol, rng)
    base, fused = _solvers(dense)
    t = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous() for k, v in seeds.items()}
    g = adjoint_lw(fused, atm_to_device(atm, torch.float32, gpu), t["flux_up"], t["flux_dn"], t["heating_rate"])
    got = {k: v.double().cpu().numpy() for k, v in g.items()}
    for key in ("tlay", "tlev", "tsfc", "h2o", "o3"):
        _check(f"dense lw d/d{key}", got[key], _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))


def test_sw_adjoint_dense_matches_fd(oracle_mod, dense, gpu):
    import torch
    from rrtmgp_b200.autodiff import adjoint_sw
    from rrtmgp_b200.solver import atm_to_device
    rng = np.random.default_rng(14)
    ncol, nlay = 2, 20
    atm = S.make_atmosphere(ncol, nlay, seed=96, clouds=True, trace_gases=True)
    atm["mu0"] = np.array([0.35, 0.8])
    kd, cl = oracle_mod.GasOptics(dense["sw"], GASES), oracle_mod.CloudOptics(dense["cloud_sw"])
    fwd = lambda a: oracle_mod.forward_sw(kd, cl, a)  # noqa: E731
    seeds = _sw_seeds(nlay, ncol, rng)
    base, fused = _solvers(dense)
    t = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous() for k, v in seeds.items()}
    g = adjoint_sw(fused, atm_to_device(atm, torch.float32, gpu), t["flux_up"], t["flux_dn"], t["flux_dn_dir"],
                   t["heating_rate"])
    got = {k: v.double().cpu().numpy() for k, v in g.items()}
    for key in ("tlay", "h2o", "o3"):
        _check(f"dense sw d/d{key}", got[key], _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))
    _check("dense sw d/dsfc_alb_dir", got["sfc_alb_dir"], _fd_bands(fwd, atm, seeds, "sfc_alb_dir"))


def test_batched_dense_matches_oracle(oracle_mod, dense, gpu):
    import torch
    from rrtmgp_b200.batch import Batched_forward
    from rrtmgp_b200.solver import atm_to_device
    grids = [(37, 23, True), (5, 128, False), (70, 129, True)]
    host = [S.make_atmosphere(n, l, seed=97 + i, clouds=True, top_at_1=top, trace_gases=True)
            for i, (n, l, top) in enumerate(grids)]
    base, _ = _solvers(dense)
    bf = Batched_forward(base, [atm_to_device(a, torch.float32, gpu) for a in host])
    got = bf.run("graph")
    torch.cuda.synchronize()
    for i, a in enumerate(host):
        rlw, rsw = _oracle(oracle_mod, dense, a)
        _check_fluxes(got[i]["lw"], rlw, f"dense batched grid {i} lw")
        _check_fluxes(got[i]["sw"], rsw, f"dense batched grid {i} sw")
    bf.close()
