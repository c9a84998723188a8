"""GPU test of the allocation-free shortwave entry point rrtmgp_b200_rte_sw_static_scratch_f32.

That entry point serves callers that cannot allocate device memory themselves (for example a
host model whose device memory belongs to its OpenACC/OpenMP runtime): it takes no workspace
and uses a scratch array compiled into the library instead.  This test calls it through the
C ABI twice in a row -- the second call reuses the scratch left by the first -- and checks
both results against the regular workspace entry point rrtmgp_b200_rte_sw_f32 with the flux
tolerance of the other GPU tests (FP32: 2e-4 relative with a floor of 1% of the largest
flux), for top-to-bottom and bottom-to-top layer orders, and that a call leaves the device's
free memory unchanged (the entry point exists for callers that cannot allocate).  It also
checks that an oversize problem is refused before anything is launched.  The file is named so
that pytest collects it after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

from rrtmgp_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _flux_err(got, ref):
    floor = 1e-2 * np.max(np.abs(ref))
    return np.max(np.abs(got - ref) / (np.abs(ref) + floor))


@pytest.mark.parametrize("top_at_1", [True, False])
def test_static_scratch_rte_sw_matches_workspace_entry_point(tables, gpu, top_at_1):
    import torch
    from rrtmgp_b200 import _abi, api

    lib = _abi.load()
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    ncol, nlay = 29, 31
    atm = S.make_atmosphere(ncol, nlay, seed=77, clouds=True, top_at_1=top_at_1)
    dt = torch.float32
    T = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=dt, device=gpu)  # noqa: E731
    g = {k: T(v.reshape(1) if v.size == 1 else v) for k, v in atm["gases"].items()}
    go = kd.gas_optics_sw(T(atm["play"]), T(atm["plev"]), T(atm["tlay"]), g)
    mu0, alb = T(atm["mu0"]), T(atm["sfc_alb_dir"])
    ref_up, ref_dn, ref_dir = api.Rte_sw.rte_sw(kd.bands, go["tau"], go["ssa"], go["g"], top_at_1, mu0,
                                                go["toa_src"], alb, alb)
    ref = [x.double().cpu().numpy() for x in (ref_up, ref_dn, ref_dir)]
    P = api._ptr
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = [[torch.full_like(ref_up, float("nan")) for _ in range(3)] for _ in range(2)]
    torch.cuda.synchronize()
    for call, (up, dn, dr) in enumerate(outs):
        free_before = torch.cuda.mem_get_info(gpu)[0]
        st = lib.rrtmgp_b200_rte_sw_static_scratch_f32(
            kd.bands.handle, ncol, nlay, int(top_at_1), P(go["tau"]), P(go["ssa"]), P(go["g"]), P(mu0),
            P(go["toa_src"]), P(alb), P(alb), None, P(up), P(dn), P(dr), stream)
        assert st == _abi.OK, lib.rrtmgp_b200_last_error()
        torch.cuda.synchronize()
        if call == 1:   # the first call may resolve the scratch address; later ones allocate nothing
            assert torch.cuda.mem_get_info(gpu)[0] == free_before
        for got, r in zip((up, dn, dr), ref):
            assert _flux_err(got.double().cpu().numpy(), r) <= 2e-4


def test_static_scratch_rejects_oversize_problem(tables, gpu):
    import torch
    from rrtmgp_b200 import _abi, api

    lib = _abi.load()
    kd = api.Gas_optics_rrtmgp(tables["sw"], S.ATM_GASES)
    ngpt = kd.get_ngpt()
    nlay = 64
    ncol = _abi.SW_STATIC_SCRATCH_MAX_ELEMS // (nlay * ngpt) + 1
    dummy = torch.empty(1, dtype=torch.float32, device=gpu)
    p = C.c_void_p(dummy.data_ptr())
    st = lib.rrtmgp_b200_rte_sw_static_scratch_f32(kd.bands.handle, ncol, nlay, 1, p, p, p, p, p, p, p, None,
                                                   p, p, p, None)
    assert st == _abi.ERR_WORKSPACE
    assert b"exceeds the built-in scratch" in lib.rrtmgp_b200_last_error()
