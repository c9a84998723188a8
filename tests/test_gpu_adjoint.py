"""Adjoint kernels against FP64 central finite differences of the oracle.

L = sum(seed_up * flux_up + seed_dn * flux_dn + seed_hr * heating_rate) with random seeds;
the FP32 adjoint gradient of every input element is compared with (L(x+h) - L(x-h)) / 2h of
the FP64 oracle forward, h = 1e-4 |x| (1e-3 |x| for the vmr fields; central differences),
wherever |x| >= 1e-5 max|x| of its field (below that the FD resolves nothing).  Columns
are independent, so one perturbation of a whole layer (or level) row gives the derivative of
every column's own loss at once.  Bound: |adjoint - FD| <= GRAD_RTOL * max |FD| of that field
(the FP32 forward itself agrees with FP64 to ~1e-5 relative; the rest is FD truncation and
the rare cell or table node crossed by the step).  Also checks the torch.autograd path.
"""
import copy

import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

pytestmark = pytest.mark.gpu
GRAD_RTOL = 3e-3
REL_STEP = 1e-4
REL_STEP_VMR = 1e-3   # tau is linear in the gas columns inside an interpolation cell


def _seeds(nlay, ncol, rng):
    return {"flux_up": rng.normal(size=(nlay + 1, ncol)), "flux_dn": rng.normal(size=(nlay + 1, ncol)),
            "heating_rate": rng.normal(size=(nlay, ncol)) * 0.1}


def _loss_cols(out, seeds):
    return sum((seeds[k] * out[k]).sum(axis=0) for k in seeds)


def _get(atm, key):
    return atm["gases"][key] if key in ("h2o", "o3") else atm[key]


def _fd(fwd, atm, seeds, key, rows=None):
    """Per-column central differences of the FP64 loss w.r.t. every element of atm[key]."""
    base = _get(atm, key)
    grad = np.zeros_like(base, dtype=np.float64)
    nrow = 1 if base.ndim == 1 else base.shape[0]
    for j in (range(nrow) if rows is None else rows):
        lp, lm = None, None
        vals = base if base.ndim == 1 else base[j]
        h = (REL_STEP_VMR if key in ("h2o", "o3") else REL_STEP) * np.maximum(np.abs(vals), 1e-30)
        for sgn in (1.0, -1.0):
            a = copy.deepcopy(atm)
            arr = _get(a, key)
            if arr.ndim == 1:
                arr += sgn * h
            else:
                arr[j] += sgn * h
            l = _loss_cols(fwd(a), seeds)
            if sgn > 0:
                lp = l
            else:
                lm = l
        g = (lp - lm) / (2 * h)
        if base.ndim == 1:
            grad[:] = g
        else:
            grad[j] = g
    return grad


def _informative(x):
    """Elements whose relative-step FD is meaningful: h2o and o3 fall to ~1e-20 (o3 to 0) near
    the model top, where a relative step moves the loss by less than the FP64 oracle resolves
    (its thin-layer source term carries ~eps/tau of noise)."""
    return np.abs(x) >= 1e-5 * np.max(np.abs(x))


def _check(name, got, ref, mask=None):
    got = np.asarray(got, np.float64)
    if mask is not None:
        got, ref = got[mask], ref[mask]
    scale = np.max(np.abs(ref))
    assert scale > 0, f"{name}: zero reference gradient"
    err = np.max(np.abs(got - ref)) / scale
    assert err <= GRAD_RTOL, f"{name}: max |adjoint - FD| / max|FD| = {err:.3e}"


def _lw_setup(tables, oracle_mod, ncol, nlay, seed, clouds, top_at_1=True):
    atm = S.make_atmosphere(ncol, nlay, seed=seed, clouds=clouds, top_at_1=top_at_1)
    kd = oracle_mod.GasOptics(tables["lw"], S.ATM_GASES)
    cl = oracle_mod.CloudOptics(tables["cloud_lw"]) if clouds else None
    return atm, (lambda a: oracle_mod.forward_lw(kd, cl, a))


def _gpu_grads(tables, atm, seeds, clouds, chunk=0):
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    fused = Fused_solver(base)
    d = atm_to_device(atm, torch.float32, "cuda")
    t = {k: torch.as_tensor(v, dtype=torch.float32, device="cuda").contiguous() for k, v in seeds.items()}
    g = adjoint_lw(fused, d, t["flux_up"], t["flux_dn"], t["heating_rate"], with_clouds=clouds, chunk=chunk)
    torch.cuda.synchronize()
    return {k: v.double().cpu().numpy() for k, v in g.items()}


@pytest.mark.parametrize("top_at_1", [True, False])
@pytest.mark.parametrize("chunk", [8, 16])
def test_lw_adjoint_matches_fd(oracle_mod, tables, gpu, top_at_1, chunk):
    rng = np.random.default_rng(3)
    ncol, nlay = 3, 24
    atm, fwd = _lw_setup(tables, oracle_mod, ncol, nlay, seed=21, clouds=True, top_at_1=top_at_1)
    seeds = _seeds(nlay, ncol, rng)
    got = _gpu_grads(tables, atm, seeds, True, chunk)
    for key in ("tlay", "tlev", "tsfc", "h2o", "o3"):
        _check(f"d/d{key}", got[key], _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))
    cloudy_l = atm["lwp"] > 0
    cloudy_i = atm["iwp"] > 0
    if cloudy_l.any():
        _check("d/dlwp", got["lwp"], _fd(fwd, atm, seeds, "lwp"), cloudy_l)
        _check("d/drel", got["rel"], _fd(fwd, atm, seeds, "rel"), cloudy_l)
    if cloudy_i.any():
        _check("d/diwp", got["iwp"], _fd(fwd, atm, seeds, "iwp"), cloudy_i)
        _check("d/drei", got["rei"], _fd(fwd, atm, seeds, "rei"), cloudy_i)


def test_lw_adjoint_deep_column_cluster(oracle_mod, tables, gpu):
    """200 layers: a cluster of two CTAs per column (128 + 72 layers), bottom-up orientation;
    FD on the rows around the CTA boundary (layers 127/128, levels 127-129) and at both ends."""
    rng = np.random.default_rng(5)
    ncol, nlay = 2, 200
    atm, fwd = _lw_setup(tables, oracle_mod, ncol, nlay, seed=25, clouds=True, top_at_1=False)
    seeds = _seeds(nlay, ncol, rng)
    got = _gpu_grads(tables, atm, seeds, True, 8)
    # rows in the reference's order (top_at_1 False: row l holds layer nlay - 1 - l from the top)
    lay_rows = sorted({0, 1, nlay - 1 - 127, nlay - 1 - 128, nlay - 2, nlay - 1})
    lev_rows = sorted({0, nlay - 127, nlay - 128, nlay - 129, nlay})
    for key, rows in (("tlay", lay_rows), ("h2o", lay_rows), ("o3", lay_rows), ("tlev", lev_rows),
                      ("tsfc", None)):
        ref = _fd(fwd, atm, seeds, key, rows)
        if rows is None:
            _check(f"d/d{key}", got[key], ref)
            continue
        mask = np.zeros_like(ref, dtype=bool)
        mask[rows] = True
        mask &= _informative(_get(atm, key))
        _check(f"d/d{key} rows {rows}", got[key], ref, mask)


def test_lw_adjoint_heating_rate_only_clear(oracle_mod, tables, gpu):
    """Seed on heating rates only (the ~0.1 Pa top layers dominate), clear sky, 60 layers."""
    rng = np.random.default_rng(4)
    ncol, nlay = 2, 60
    atm, fwd = _lw_setup(tables, oracle_mod, ncol, nlay, seed=22, clouds=False)
    seeds = {"heating_rate": rng.normal(size=(nlay, ncol))}
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    d = atm_to_device(atm, torch.float32, "cuda")
    g = adjoint_lw(Fused_solver(base), d, None, None,
                   torch.as_tensor(seeds["heating_rate"], dtype=torch.float32, device="cuda"), with_clouds=False)
    for key in ("tlay", "h2o", "o3", "tlev"):
        _check(f"HR d/d{key}", g[key].double().cpu().numpy(), _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))


def test_lw_autograd_directional(oracle_mod, tables, gpu):
    """torch.autograd through the fused forward: grad . v against a directional central FD."""
    import torch
    from rrtmgp_b200.autodiff import longwave
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    rng = np.random.default_rng(5)
    ncol, nlay = 16, 40
    atm, fwd = _lw_setup(tables, oracle_mod, ncol, nlay, seed=23, clouds=True)
    seeds = _seeds(nlay, ncol, rng)
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    fused = Fused_solver(base)
    d = atm_to_device(atm, torch.float32, "cuda")
    leaves = [d["tlay"], d["tlev"], d["tsfc"], d["gases"]["h2o"], d["gases"]["o3"]]
    for t in leaves:
        t.requires_grad_(True)
    out = longwave(fused, d)
    loss = sum((torch.as_tensor(seeds[k], dtype=torch.float32, device="cuda") * out[k]).sum() for k in seeds)
    loss.backward()
    dirs = {"tlay": rng.normal(size=atm["tlay"].shape), "tlev": rng.normal(size=atm["tlev"].shape),
            "tsfc": rng.normal(size=atm["tsfc"].shape), "h2o": rng.normal(size=atm["gases"]["h2o"].shape),
            "o3": rng.normal(size=atm["gases"]["o3"].shape)}
    scale = {"tlay": 1e-2, "tlev": 1e-2, "tsfc": 1e-2, "h2o": 1e-4, "o3": 1e-4}   # relative step per field
    ad = 0.0
    for key, t in zip(("tlay", "tlev", "tsfc", "h2o", "o3"), leaves):
        ad += float((t.grad.double().cpu().numpy() * dirs[key] * scale[key] * np.abs(_get(atm, key))).sum())

    def shifted(eps):
        a = copy.deepcopy(atm)
        for key in dirs:
            arr = _get(a, key)
            arr += eps * dirs[key] * scale[key] * np.abs(arr)
        return _loss_cols(fwd(a), seeds).sum()

    eps = 1e-3
    fd = (shifted(eps) - shifted(-eps)) / (2 * eps)
    assert abs(ad - fd) <= 2e-3 * abs(fd), f"directional derivative: autograd {ad:.6e} vs FD {fd:.6e}"


# ---------------------------------------------------------------------------------------------
# Shortwave
# ---------------------------------------------------------------------------------------------
def _sw_setup(tables, oracle_mod, ncol, nlay, seed, clouds, top_at_1=True):
    rng = np.random.default_rng(seed)
    atm = S.make_atmosphere(ncol, nlay, seed=seed, clouds=clouds, top_at_1=top_at_1)
    nb = atm["sfc_alb_dir"].shape[1]
    atm["sfc_alb_dir"] = rng.uniform(0.05, 0.6, (ncol, nb))
    atm["sfc_alb_dif"] = rng.uniform(0.05, 0.6, (ncol, nb))
    atm["mu0"] = np.linspace(0.15, 0.95, ncol)
    kd = oracle_mod.GasOptics(tables["sw"], S.ATM_GASES)
    cl = oracle_mod.CloudOptics(tables["cloud_sw"]) if clouds else None
    return atm, (lambda a: oracle_mod.forward_sw(kd, cl, a))


def _sw_seeds(nlay, ncol, rng):
    s = _seeds(nlay, ncol, rng)
    s["flux_dn_dir"] = rng.normal(size=(nlay + 1, ncol))
    return s


def _fd_bands(fwd, atm, seeds, key):
    """Per-column FD w.r.t. each band of a (ncol, nband) surface field."""
    base = atm[key]
    grad = np.zeros_like(base)
    for b in range(base.shape[1]):
        h = REL_STEP * np.abs(base[:, b])
        ls = []
        for sgn in (1.0, -1.0):
            a = copy.deepcopy(atm)
            a[key][:, b] += sgn * h
            ls.append(_loss_cols(fwd(a), seeds))
        grad[:, b] = (ls[0] - ls[1]) / (2 * h)
    return grad


def _gpu_grads_sw(tables, atm, seeds, clouds):
    import torch
    from rrtmgp_b200.autodiff import adjoint_sw
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    d = atm_to_device(atm, torch.float32, "cuda")
    t = {k: torch.as_tensor(v, dtype=torch.float32, device="cuda").contiguous() for k, v in seeds.items()}
    g = adjoint_sw(Fused_solver(base), d, t.get("flux_up"), t.get("flux_dn"), t.get("flux_dn_dir"),
                   t.get("heating_rate"), with_clouds=clouds)
    torch.cuda.synchronize()
    return {k: v.double().cpu().numpy() for k, v in g.items()}


@pytest.mark.parametrize("nlay", [24, 80])   # 80 layers: a cluster of two CTAs per column
@pytest.mark.parametrize("top_at_1", [True, False])
def test_sw_adjoint_matches_fd(oracle_mod, tables, gpu, nlay, top_at_1):
    rng = np.random.default_rng(6)
    ncol = 3
    atm, fwd = _sw_setup(tables, oracle_mod, ncol, nlay, seed=31 + nlay, clouds=True, top_at_1=top_at_1)
    seeds = _sw_seeds(nlay, ncol, rng)
    got = _gpu_grads_sw(tables, atm, seeds, True)
    for key in ("tlay", "h2o", "o3"):
        _check(f"sw d/d{key}", got[key], _fd(fwd, atm, seeds, key), _informative(_get(atm, key)))
    for key in ("sfc_alb_dir", "sfc_alb_dif"):
        _check(f"sw d/d{key}", got[key], _fd_bands(fwd, atm, seeds, key))
    cloudy_l, cloudy_i = atm["lwp"] > 0, atm["iwp"] > 0
    if cloudy_l.any():
        _check("sw d/dlwp", got["lwp"], _fd(fwd, atm, seeds, "lwp"), cloudy_l)
        _check("sw d/drel", got["rel"], _fd(fwd, atm, seeds, "rel"), cloudy_l)
    if cloudy_i.any():
        _check("sw d/diwp", got["iwp"], _fd(fwd, atm, seeds, "iwp"), cloudy_i)
        _check("sw d/drei", got["rei"], _fd(fwd, atm, seeds, "rei"), cloudy_i)


@pytest.mark.parametrize("nlay", [24, 80])
def test_sw_adjoint_resonance_columns(oracle_mod, tables, gpu, nlay):
    """Columns with mu0 near 1/k of the strongly absorbing g-points (k ~ 2): 13% of the (layer,
    g-point) pairs at mu0 = 0.5 take the factored k mu0 = 1 form of the two-stream
    (|1 - (k mu0)^2| < 0.02) and its hand-written reverse mode.  Checked per column against
    FP64 central differences."""
    rng = np.random.default_rng(8)
    ncol = 4
    atm, fwd = _sw_setup(tables, oracle_mod, ncol, nlay, seed=57 + nlay, clouds=True)
    atm["mu0"] = np.array([0.4995, 0.501, 0.51, 0.55])
    seeds = _sw_seeds(nlay, ncol, rng)
    got = _gpu_grads_sw(tables, atm, seeds, True)
    for key in ("tlay", "h2o", "o3"):
        ref = _fd(fwd, atm, seeds, key)
        inf = _informative(_get(atm, key))
        for c in range(ncol):
            _check(f"sw d/d{key} column {c}", got[key][:, c], ref[:, c], inf[:, c])


def test_sw_autograd_directional(oracle_mod, tables, gpu):
    import torch
    from rrtmgp_b200.autodiff import shortwave
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    rng = np.random.default_rng(7)
    ncol, nlay = 16, 40
    atm, fwd = _sw_setup(tables, oracle_mod, ncol, nlay, seed=41, clouds=True)
    seeds = _sw_seeds(nlay, ncol, rng)
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    d = atm_to_device(atm, torch.float32, "cuda")
    leaves = [d["tlay"], d["gases"]["h2o"], d["gases"]["o3"]]
    for t in leaves:
        t.requires_grad_(True)
    out = shortwave(Fused_solver(base), d)
    loss = sum((torch.as_tensor(seeds[k], dtype=torch.float32, device="cuda") * out[k]).sum() for k in seeds)
    loss.backward()
    dirs = {k: rng.normal(size=_get(atm, k).shape) for k in ("tlay", "h2o", "o3")}
    scale = {"tlay": 1e-2, "h2o": 1e-3, "o3": 1e-3}
    ad = sum(float((t.grad.double().cpu().numpy() * dirs[k] * scale[k] * np.abs(_get(atm, k))).sum())
             for k, t in zip(("tlay", "h2o", "o3"), leaves))

    def shifted(eps):
        a = copy.deepcopy(atm)
        for k in dirs:
            arr = _get(a, k)
            arr += eps * dirs[k] * scale[k] * np.abs(arr)
        return _loss_cols(fwd(a), seeds).sum()

    eps = 1e-3
    fd = (shifted(eps) - shifted(-eps)) / (2 * eps)
    assert abs(ad - fd) <= 2e-3 * abs(fd), f"directional derivative: autograd {ad:.6e} vs FD {fd:.6e}"


@pytest.mark.parametrize("nlay", [60, 200])
def test_forward_adjoint_one_launch(tables, gpu, nlay):
    """rrtmgp_b200_forward_adjoint_{lw,sw}_f32: the fluxes equal the fused forward's and the
    gradients the adjoint-only launch's, to FP32 rounding (the same arithmetic compiled into
    another kernel), for one CTA (60 layers) and a cluster of CTAs (200 layers)."""
    import torch
    from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device
    base = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    fused = Fused_solver(base)
    ncol = 40
    atm = atm_to_device(S.make_atmosphere(ncol, nlay, seed=71, clouds=True, top_at_1=nlay < 100), torch.float32, "cuda")
    g = torch.Generator(device="cuda").manual_seed(3)
    sd = {k: torch.randn(shape, generator=g, device="cuda") for k, shape in
          (("up", (nlay + 1, ncol)), ("dn", (nlay + 1, ncol)), ("dir", (nlay + 1, ncol)), ("hr", (nlay, ncol)))}
    for dom in ("lw", "sw"):
        if dom == "lw":
            ref_f = {k: v.clone() for k, v in fused.solve_lw(atm).items()}
            ref_g = adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"])
            f, gr = adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"], with_fluxes=True)
        else:
            ref_f = {k: v.clone() for k, v in fused.solve_sw(atm).items()}
            ref_g = adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"])
            f, gr = adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"], with_fluxes=True)
        torch.cuda.synchronize()
        for k in ref_f:
            d = float((f[k] - ref_f[k]).abs().max())
            assert torch.isfinite(f[k]).all() and d < 2e-3, f"{dom} {k}: {d:.3e}"
        for k in ref_g:
            scale = float(ref_g[k].abs().max()) + 1e-30
            d = float((gr[k] - ref_g[k]).abs().max()) / scale
            assert d < 1e-4, f"{dom} grad {k}: {d:.3e}"
