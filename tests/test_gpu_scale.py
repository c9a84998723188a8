"""Parity at the benchmark sizes: the fused FP32 kernels run on whole benchmark grids and a
subsample of columns spread over each grid is compared with the FP64 oracle.

  * 8192 x 128 all-sky (the forward benchmark's grid and seed): every 32nd column;
  * 262144 x 256 all-sky, built in 16384-column blocks as the deep-column benchmark builds it:
    16 columns from each of four blocks spread over the grid (first, two inner, last), for the
    fused forward and for the fluxes of the forward + adjoint launches;
  * 4096 x 128 all-sky forward + adjoint with every output seeded: the gradients of 8 sampled
    columns against FP64 central differences of the oracle.

Bounds are the FP32 product's stated ones: 0.05 W/m2 for every flux level and 0.01 K/day for
every heating-rate layer; gradients as the other adjoint tests (3e-3 of max|FD| per field),
plus a per-element check where the derivative is large (|FD| >= 5% of the field's max: 1%
relative), which a mis-signed or mis-scaled term would fail.
"""
import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

from test_gpu_adjoint import GRAD_RTOL, _fd, _get, _informative

pytestmark = pytest.mark.gpu
FLUX_TOL = 0.05
HR_TOL = 0.01


def _solvers(tables):
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    return base, Fused_solver(base)


def _oracles(oracle_mod, tables):
    glw, gsw = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES), oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    clw, csw = oracle_mod.CloudOptics(tables["cloud_lw"]), oracle_mod.CloudOptics(tables["cloud_sw"])
    return (lambda a: oracle_mod.forward_lw(glw, clw, a)), (lambda a: oracle_mod.forward_sw(gsw, csw, a))


def _compare(got, ref, cols, what):
    """got: device fluxes of the whole grid; ref: oracle fluxes of the columns `cols`."""
    worst = {}
    for k in ref:
        if k not in got:
            continue
        g = got[k][:, cols].double().cpu().numpy()
        e = float(np.max(np.abs(g - ref[k])))
        worst[k] = e
        tol = HR_TOL if k == "heating_rate" else FLUX_TOL
        assert e <= tol, f"{what} {k}: {e:.3e} > {tol}"
    return worst


def test_config2_grid_fused_forward_matches_oracle(oracle_mod, tables, gpu):
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, fused = _solvers(tables)
    atm = S.make_atmosphere(8192, 128, seed=42, clouds=True)
    d = atm_to_device(atm, torch.float32, gpu)
    lw, sw = fused.solve_lw(d), fused.solve_sw(d)
    torch.cuda.synchronize()
    cols = np.arange(0, 8192, 32)
    host = _take(atm, cols)
    olw, osw = _oracles(oracle_mod, tables)
    _compare(lw, olw(host), cols, "8192x128 lw")
    _compare(sw, osw(host), cols, "8192x128 sw")


def test_config2_grid_staged_fp32_matches_oracle(oracle_mod, tables, gpu):
    """The class-API sequence in FP32 on the whole 8192 x 128 grid: gas optics on the packed
    tables, the TMA-staged longwave solver, the chunked shortwave solver, broadband sums and
    heating rates from absorbed flux; every 32nd column against the oracle."""
    import torch
    from rrtmgp_b200.solver import atm_to_device
    base, _ = _solvers(tables)
    atm = S.make_atmosphere(8192, 128, seed=42, clouds=True)
    d = atm_to_device(atm, torch.float32, gpu)
    top = bool(atm["play"][0, 0] < atm["play"][-1, 0])
    lw, sw = base.solve_lw(d, top_at_1=top), base.solve_sw(d, top_at_1=top)
    torch.cuda.synchronize()
    cols = np.arange(0, 8192, 32)
    host = _take(atm, cols)
    olw, osw = _oracles(oracle_mod, tables)
    _compare(lw, olw(host), cols, "staged 8192x128 lw")
    _compare(sw, osw(host), cols, "staged 8192x128 sw")


def _take(atm, cols):
    """The columns `cols` (any index array) of a host atmosphere."""
    out = {}
    ncol = atm["ncol"]
    for k, v in atm.items():
        if k == "gases":
            out[k] = {g: (a[:, cols] if a.ndim == 2 and a.shape[1] == ncol and ncol > 1 else a) for g, a in v.items()}
        elif k == "ncol":
            out[k] = len(cols)
        elif not hasattr(v, "ndim"):
            out[k] = v
        elif k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif") or (v.ndim == 1 and v.shape[0] == ncol):
            out[k] = np.ascontiguousarray(v[cols])
        elif v.ndim == 2 and v.shape[1] == ncol:
            out[k] = np.ascontiguousarray(v[:, cols])
        else:
            out[k] = v
    return out


def test_config5_grid_forward_and_adjoint_fluxes_match_oracle(oracle_mod, tables, gpu):
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
    from rrtmgp_b200.solver import atm_to_device
    ncol, nlay, blk, seed = 262144, 256, 16384, 47
    base, fused = _solvers(tables)
    atm = None
    picks = {0: None, 5 * blk: None, 11 * blk: None, ncol - blk: None}
    rng = np.random.default_rng(3)
    for c0 in range(0, ncol, blk):
        host = S.make_atmosphere(blk, nlay, seed=seed + c0, clouds=True)
        if c0 in picks:
            picks[c0] = (np.sort(rng.choice(blk, 16, replace=False)), host)
        part = atm_to_device(host, torch.float32, gpu)
        if atm is None:
            atm = {k: torch.empty(v.shape[:-1] + (ncol,), dtype=v.dtype, device=gpu)
                   for k, v in part.items() if k not in ("gases", "emis_sfc", "sfc_alb_dir", "sfc_alb_dif")}
            for k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif"):
                atm[k] = torch.empty((ncol,) + part[k].shape[1:], dtype=torch.float32, device=gpu)
            atm["gases"] = {k: (torch.empty(v.shape[:-1] + (ncol,), dtype=v.dtype, device=gpu) if v.numel() > 1
                                else v.clone()) for k, v in part["gases"].items()}
        for k, v in part.items():
            if k == "gases":
                for g, t in v.items():
                    if t.numel() > 1:
                        atm["gases"][g][:, c0:c0 + blk].copy_(t)
            elif k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif"):
                atm[k][c0:c0 + blk].copy_(v)
            else:
                atm[k][..., c0:c0 + blk].copy_(v)
        del part
    lw = {k: v.clone() for k, v in fused.solve_lw(atm).items()}
    sw = {k: v.clone() for k, v in fused.solve_sw(atm).items()}
    gen = torch.Generator(device=gpu).manual_seed(5)
    sd = {k: torch.randn(shape, generator=gen, device=gpu) for k, shape in
          (("up", (nlay + 1, ncol)), ("dn", (nlay + 1, ncol)), ("dir", (nlay + 1, ncol)), ("hr", (nlay, ncol)))}
    alw = adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"], with_fluxes=True)[0]
    asw = adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"], with_fluxes=True)[0]
    torch.cuda.synchronize()
    olw, osw = _oracles(oracle_mod, tables)
    for c0, (cols, host) in picks.items():
        sub = _take(host, cols)
        rlw, rsw = olw(sub), osw(sub)
        g = c0 + cols
        _compare(lw, rlw, g, f"262144x256 lw block {c0}")
        _compare(sw, rsw, g, f"262144x256 sw block {c0}")
        _compare(alw, rlw, g, f"262144x256 forward+adjoint lw block {c0}")
        _compare(asw, rsw, g, f"262144x256 forward+adjoint sw block {c0}")


@pytest.mark.parametrize("domain", ["lw", "sw"])
def test_config4_grid_adjoint_matches_fd_on_sampled_columns(oracle_mod, tables, gpu, domain):
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
    from rrtmgp_b200.solver import atm_to_device
    ncol, nlay = 4096, 128
    base, fused = _solvers(tables)
    atm = S.make_atmosphere(ncol, nlay, seed=44, clouds=True)
    rng = np.random.default_rng(9)
    seeds = {"flux_up": rng.normal(size=(nlay + 1, ncol)), "flux_dn": rng.normal(size=(nlay + 1, ncol)),
             "heating_rate": rng.normal(size=(nlay, ncol)) * 0.1}
    if domain == "sw":
        seeds["flux_dn_dir"] = rng.normal(size=(nlay + 1, ncol))
    t = {k: torch.as_tensor(v, dtype=torch.float32, device=gpu).contiguous() for k, v in seeds.items()}
    d = atm_to_device(atm, torch.float32, gpu)
    if domain == "lw":
        g = adjoint_lw(fused, d, t["flux_up"], t["flux_dn"], t["heating_rate"])
    else:
        g = adjoint_sw(fused, d, t["flux_up"], t["flux_dn"], t["flux_dn_dir"], t["heating_rate"])
    torch.cuda.synchronize()
    cols = np.sort(rng.choice(ncol, 8, replace=False))
    host = _take(atm, cols)
    sub_seeds = {k: v[:, cols] for k, v in seeds.items()}
    olw, osw = _oracles(oracle_mod, tables)
    fwd = olw if domain == "lw" else osw
    keys = ("tlay", "tlev", "tsfc", "h2o", "o3") if domain == "lw" else ("tlay", "h2o", "o3")
    for key in keys:
        ref = _fd(fwd, host, sub_seeds, key)
        got = g[key].double().cpu().numpy()
        got = got[cols] if got.ndim == 1 else got[:, cols]
        mask = _informative(_get(host, key))
        diff = np.abs(got - ref)[mask]
        scale = np.max(np.abs(ref[mask]))
        assert np.max(diff) <= GRAD_RTOL * scale, f"{domain} d/d{key}: {np.max(diff) / scale:.3e} of max|FD|"
        big = np.abs(ref) >= 0.05 * scale
        big &= mask
        rel = np.abs(got - ref)[big] / np.abs(ref[big])
        assert np.max(rel) <= 1e-2, f"{domain} d/d{key}: large derivatives off by {np.max(rel):.3e} relative"
