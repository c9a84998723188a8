#!/usr/bin/env python
"""Throughput benchmark of the B200 column-radiation path: all-sky LW + SW forward.

Metric: columns/s (one column = gas optics + cloud optics + solver + broadband reduction +
heating rates for LW 256 and SW 224 g-points over nlay layers), FP32, synthetic seeded
atmospheres and tables with the reference schema (the real RRTMGP tables are not available).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--path fused|staged] [--ncol C] [--nlay L]

--path fused (default) runs the product path: one fused kernel per LW and per SW solve.
--path staged runs the reference-shaped per-stage kernels over (g, lay, col) arrays.

One process per GPU (torchrun for N > 1); columns are sharded across ranks with no exchange
(weak scaling: every rank owns ncol columns).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path[:0] = [str(REPO), str(REPO / "rte-rrtmgp-cpp_b200")]

import numpy as np  # noqa: E402

METRIC = "columns/s (all-sky LW+SW, 1 B200) plain FP64 vs FP32+adjoint at stated W/m2 err"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu-child"])
    ap.add_argument("--path", default="fused", choices=["staged", "fused"])
    ap.add_argument("--ncol", type=int, default=8192)
    ap.add_argument("--nlay", type=int, default=128)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--batched-grids", type=int, default=512,
                    help="uneven-grid batch: grids with ncol U{64..4096}, nlay U{40..200} (0: skip)")
    ap.add_argument("--batched-steps", type=int, default=3)
    ap.add_argument("--batched-no-autotune", action="store_true",
                    help="use the built-in tile-shape heuristic instead of the autotuner")
    ap.add_argument("--deep-ncol", type=int, default=262144,
                    help="deep-column forward + adjoint: ncol (0: skip)")
    ap.add_argument("--deep-nlay", type=int, default=256)
    ap.add_argument("--deep-steps", type=int, default=2)
    return ap.parse_args()


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        lines = Path(self.file.name).read_text().strip().splitlines()
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def bytes_per_column(nlay, glw=256, gsw=224, nb_lw=16, nb_sw=14, B=4):
    """Algorithmic HBM bytes per column of each staged kernel (inputs read once, outputs
    written once; k-tables are L2 resident and counted zero)."""
    L, V = nlay, nlay + 1
    return {
        "gas_optics_lw": ((6 * L + 3) + 4 * L * glw + 2 * glw) * B,
        "gas_optics_sw": ((4 * L + 1) + 3 * L * gsw) * B,
        "lw_solver": (4 * L * glw + glw + nb_lw + 2 * V * glw) * B,
        "sw_solver": (3 * L * gsw + 1 + gsw + 2 * nb_sw + 3 * V * gsw) * B,
        "broadband_lw": (2 * V * glw + 3 * V) * B,
        "broadband_sw": (3 * V * gsw + 4 * V) * B,
        "cloud_lw": (4 * L + L * nb_lw) * B,
        "cloud_sw": (4 * L + 3 * L * nb_sw) * B,
        "add_to_lw": (2 * L * glw + L * nb_lw) * B,
        "add_to_sw": (6 * L * gsw + 3 * L * nb_sw) * B,
        "delta_sw": (6 * L * nb_sw) * B,
        "heating": (4 * V + L) * B * 2,
    }


def fused_flops_per_column(nlay, glw=256, gsw=224):
    """Algorithmic FP32 FLOPs (FMA = 2) per column of the fused kernels, counted from the
    kernel source per (layer, g-point): LW 79 (major 16, minor 10, cloud 1, Planck fraction 16,
    sources 3, layer terms 15, chunk maps 7, pass 2 8, reduction 3) plus 1 exp and 1 divide;
    SW 210 (major 16, minor 10, Rayleigh 9, combine 7, two-stream 108, adding composite 26,
    direct outputs 4, passes 2/3 26, reduction 4) plus 1 sqrt, 2 exp and 6 divides.
    Transcendentals and divides are not counted as FLOPs."""
    return {"lw_forward_kernel": 79 * nlay * glw, "sw_forward_kernel": 210 * nlay * gsw}


def fused_bytes_per_column(nlay, nb_lw=16, nb_sw=14, B=4):
    """HBM bytes per column the fused kernels must move: inputs once, outputs once.  Inputs:
    play, tlay, plev (+ tlev, tsfc for LW), lwp/iwp/rel/rei, the h2o and o3 fields (the other
    gases are scalars), emissivity or mu0/tsi/albedos; outputs: the level fluxes and the
    layer heating rates."""
    L, V = nlay, nlay + 1
    lw_in = (2 * L + 2 * V + 1 + 4 * L + 2 * L + nb_lw) * B
    lw_out = (3 * V + L) * B
    sw_in = (2 * L + V + 4 * L + 2 * L + 2 + 2 * nb_sw) * B
    sw_out = (4 * V + L) * B
    return {"lw_forward_kernel": lw_in + lw_out, "sw_forward_kernel": sw_in + sw_out}


def fp32_peak(torch, dev, stream):
    """FP32 FMA throughput of this GPU measured with the library's FMA probe (TFLOP/s)."""
    from rrtmgp_b200 import _abi
    lib = _abi.load()
    import ctypes as C
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, iters = nsm * 4, 4096
    out = torch.empty(blocks, dtype=torch.float32, device=dev)
    s = C.c_void_p(stream.cuda_stream)
    for _ in range(2):
        _abi.check(lib.rrtmgp_b200_fp32_fma_probe(blocks, iters, C.c_void_p(out.data_ptr()), s))
    best = None
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _abi.check(lib.rrtmgp_b200_fp32_fma_probe(blocks, iters, C.c_void_p(out.data_ptr()), s))
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    return blocks * 512.0 * iters * 256.0 / (best * 1e-3) / 1e12


def ncu_traffic():
    """dram bytes per column of each kernel from the committed ncu summary, if any."""
    p = REPO / "profiles" / "ncu_traffic.txt"
    out = {}
    if p.exists():
        for ln in p.read_text().splitlines():
            parts = ln.split()
            if len(parts) >= 2 and not ln.startswith("#"):
                try:
                    out[parts[0]] = float(parts[1])
                except ValueError:
                    pass
    return out


def cpu_baseline(args, tables, seconds):
    """The oracle (FP64 C++ port of the reference path) on the host cores."""
    from oracle import oracle as O
    from rrtmgp_b200 import synthetic as S
    ncores = os.cpu_count() or 1
    O.set_threads(ncores)
    klw = O.GasOptics(tables["lw"], S.ATM_GASES)
    ksw = O.GasOptics(tables["sw"], S.ATM_GASES)
    clw = O.CloudOptics(tables["cloud_lw"])
    csw = O.CloudOptics(tables["cloud_sw"])

    def run(nc):
        atm = S.make_atmosphere(nc, args.nlay, seed=args.seed, clouds=True)
        t0 = time.perf_counter()
        O.forward_lw(klw, clw, atm)
        O.forward_sw(ksw, csw, atm)
        return time.perf_counter() - t0

    probe = 64
    dt = run(probe)
    nc = int(min(args.ncol, max(probe, probe * seconds / max(dt, 1e-6) / 2)))
    reps, tot = 0, 0.0
    while tot < seconds * 0.5 or reps < 1:
        tot += run(nc)
        reps += 1
    return {"value": reps * nc / tot, "unit": "columns/s", "cores": ncores, "kind": "port",
            "sample": f"{reps} x {nc} columns of the {args.nlay}-layer all-sky LW+SW forward, FP64, "
                      f"OpenMP over columns"}


def run_reference_gpu_child(args):
    """Child process of the reference arm: the reference's own FP64 CUDA classes
    (oracle/_ref, built from the reference sources) timed on the all-sky forward of this
    workload as its test driver runs it (solve_gpu, columns in blocks of 1024), and checked
    on 64 sampled columns against the CPU port.  Prints one JSON object.  Runs in its own
    working directory because the reference's tuner reads and rewrites a cache file there."""
    from oracle import oracle as O
    from oracle import ref_gpu
    from rrtmgp_b200 import synthetic as S
    tables = {"lw": S.make_kdist("lw"), "sw": S.make_kdist("sw"),
              "cloud_lw": S.make_cloud_luts("lw"), "cloud_sw": S.make_cloud_luts("sw")}
    atm = S.make_atmosphere(args.ncol, args.nlay, seed=args.seed, clouds=True)
    ref_gpu.write_tuning(Path.cwd())
    lib = ref_gpu.load()
    ms_lw, ms_sw, out = ref_gpu.time_forward(lib, tables, atm, nsteps=max(3, args.steps // 5 + 1))
    cols = np.linspace(0, args.ncol - 1, 64).astype(int)
    sub = {k: (v[:, cols] if getattr(v, "ndim", 0) == 2 and v.shape[1] == args.ncol and
               k not in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif") else
               (v[cols] if getattr(v, "ndim", 0) >= 1 and v.shape[0] == args.ncol else v))
           for k, v in atm.items() if k != "gases"}
    sub["gases"] = {k: (v[:, cols] if v.size > 1 else v) for k, v in atm["gases"].items()}
    sub["ncol"] = len(cols)
    rlw = O.forward_lw(O.GasOptics(tables["lw"], S.ATM_GASES), O.CloudOptics(tables["cloud_lw"]), sub)
    rsw = O.forward_sw(O.GasOptics(tables["sw"], S.ATM_GASES), O.CloudOptics(tables["cloud_sw"]), sub)
    err = max(float(np.max(np.abs(out[d + "_" + k][:, cols] - r["flux_" + k])))
              for d, r in (("lw", rlw), ("sw", rsw)) for k in ("up", "dn"))
    ms = ms_lw + ms_sw
    print(json.dumps({"value": args.ncol / (ms * 1e-3), "unit": "columns/s", "ms_per_step": ms,
                      "kernel_ms": {"lw": round(ms_lw, 3), "sw": round(ms_sw, 3)}, "dtype": "f64",
                      "max_flux_diff_vs_cpu_port_w_m2": err,
                      "how": "the reference's Gas_optics_rrtmgp_gpu, Cloud_optics_gpu, Rte_lw_gpu, Rte_sw_gpu and "
                             "Fluxes_broadband_gpu built from its sources (FP64), columns in blocks of 1024 as its "
                             "solve_gpu, tuner cache pre-seeded (no tuning)"}), flush=True)
    return 0


def reference_gpu(args):
    """Secondary measurement of the reference arm: the reference's GPU forward (FP64), run in a
    child process; an {"unavailable": ...} object when it cannot run here."""
    lib = REPO / "oracle" / "_ref" / "libref_rrtmgp_f64.so"
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
    except Exception as e:   # noqa: BLE001
        return {"unavailable": f"torch: {e}"}
    if not lib.exists():
        return {"unavailable": "oracle/_ref/libref_rrtmgp_f64.so not built (the reference sources are needed)"}
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [sys.executable, str(REPO / "bench.py"), "--impl", "reference-gpu-child", "--ncol", str(args.ncol),
               "--nlay", str(args.nlay), "--seed", str(args.seed), "--steps", str(args.steps)]
        try:
            r = subprocess.run(cmd, cwd=tmp, capture_output=True, text=True, timeout=900)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference GPU run exceeded 900 s"}
        if r.returncode != 0:
            return {"unavailable": "reference GPU run failed: " + (r.stderr.strip().splitlines() or ["?"])[-1][:200]}
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        return json.loads(lines[-1]) if lines else {"unavailable": "no output from the reference GPU run"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from rrtmgp_b200 import synthetic as S
    tables = {"lw": S.make_kdist("lw"), "sw": S.make_kdist("sw"),
              "cloud_lw": S.make_cloud_luts("lw"), "cloud_sw": S.make_cloud_luts("sw")}
    from oracle import oracle as O
    ncores = os.cpu_count() or 1
    O.set_threads(ncores)
    klw = O.GasOptics(tables["lw"], S.ATM_GASES)
    ksw = O.GasOptics(tables["sw"], S.ATM_GASES)
    clw = O.CloudOptics(tables["cloud_lw"])
    csw = O.CloudOptics(tables["cloud_sw"])
    # Bounded sample per step so that warmup + steps finish within a few minutes.
    nc = min(args.ncol, 512)
    atm = S.make_atmosphere(nc, args.nlay, seed=args.seed, clouds=True)
    for _ in range(args.warmup):
        O.forward_lw(klw, clw, atm)
        O.forward_sw(ksw, csw, atm)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.forward_lw(klw, clw, atm)
        O.forward_sw(ksw, csw, atm)
    dt = (time.perf_counter() - t0) / args.steps
    value = nc / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"all-sky LW+SW forward, ncol={args.ncol}, nlay={args.nlay}", "ncol": args.ncol,
                   "nlay": args.nlay, "sample_ncol_per_step": nc},
        "cpu_baseline": {"value": value, "unit": "columns/s", "cores": ncores, "kind": "port",
                         "sample": f"{nc} columns per step of the {args.nlay}-layer all-sky LW+SW forward "
                                   f"(FP64 C++ restatement of the reference path; the reference's own CPU "
                                   f"build needs the absent rte-rrtmgp Fortran, gfortran, netCDF and Boost)"},
        "e2e": {"value": value, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu(args),
    }
    print(json.dumps(line), flush=True)
    return 0


def batched_bench(args, solver, dev, stream, flush, rank, world, dist):
    """Uneven batch: args.batched_grids all-sky grids, ncol U{64..4096}, nlay U{40..200}, LW+SW
    forward of all of them per step; one persistent launch replayed from a captured CUDA graph
    (tile shapes autotuned) against one fused launch per grid and domain."""
    import torch
    from rrtmgp_b200 import shard
    from rrtmgp_b200 import synthetic as S
    from rrtmgp_b200.batch import Batched_forward
    from rrtmgp_b200.solver import atm_to_device

    rng = np.random.default_rng(shard.rank_seed(args.seed + 3, rank))
    ncols = rng.integers(64, 4097, args.batched_grids)
    nlays = rng.integers(40, 201, args.batched_grids)
    atms = [atm_to_device(S.make_atmosphere(int(c), int(l), seed=int(rng.integers(1 << 30)), clouds=True),
                          torch.float32, dev) for c, l in zip(ncols, nlays)]
    bf = Batched_forward(solver, atms)
    t0 = time.perf_counter()
    plan = bf.plan() if args.batched_no_autotune else bf.autotune(reps=2)
    tune_s = time.perf_counter() - t0
    res = {}
    outs = {}
    for mode in ("graph", "per_grid"):
        for _ in range(2):
            bf.run(mode)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.batched_steps)]
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            bf.run(mode)
            e1.record(stream)
        torch.cuda.synchronize()
        ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
        ms = shard.max_over_ranks(ms, dist if world > 1 else None, dev)
        res[mode] = {"value": bf.columns() * world / (ms * 1e-3), "unit": "columns/s", "ms_per_step": ms}
        outs[mode] = [{d: {k: v.clone() for k, v in o[d].items()} for d in o} for o in bf.out]
    # The autotuned shapes may use another chunk length than the per-grid rule: FP32-level
    # differences only.
    dflux = max(float((a[d][k] - b[d][k]).abs().max()) for a, b in zip(outs["graph"], outs["per_grid"])
                for d in a for k in a[d] if k != "heating_rate")
    dhr = max(float((a[d]["heating_rate"] - b[d]["heating_rate"]).abs().max())
              for a, b in zip(outs["graph"], outs["per_grid"]) for d in a)
    st = bf.stats()
    nl = np.asarray(nlays)
    nc = np.asarray(ncols)
    out = {"workload": f"{args.batched_grids} all-sky grids, ncol U{{64..4096}}, nlay U{{40..200}}, LW+SW forward",
           "columns": bf.columns(), "mean_nlay": float((nc * nl).sum() / nc.sum()),
           "persistent_graph": res["graph"], "per_grid_launches": res["per_grid"],
           "speedup": res["per_grid"]["ms_per_step"] / res["graph"]["ms_per_step"],
           "autotune_s": tune_s, "tiles": st["tiles"], "ctas": st["ctas"], "smem_bytes": st["smem_bytes"],
           "launches_per_step": {"persistent_graph": st["launches_persistent"],
                                 "per_grid": st["launches_per_grid"]},
           "plan": {f"{'lw' if d == 0 else 'sw'}{8 * b - 7}-{8 * b}": list(v[:2]) for (d, b), v in plan.items()},
           "max_diff_vs_per_grid": {"flux_w_m2": dflux, "heating_rate_k_day": dhr}}
    bf.close()
    del atms, outs
    return out


def deep_bench(args, solver, fused, dev, stream, flush, rank, world, dist):
    """Deep columns: args.deep_ncol all-sky columns of args.deep_nlay layers, FP32 forward +
    adjoint (LW and SW, every output seeded) per step, against the plain FP64 GPU forward of
    this build run in blocks of 8192 columns (its g-point arrays of the whole grid would not fit)."""
    import torch
    from rrtmgp_b200 import shard
    from rrtmgp_b200 import synthetic as S
    from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
    from rrtmgp_b200.solver import atm_to_device

    ncol, nlay = args.deep_ncol, args.deep_nlay
    blk = 16384
    atm = None
    for c0 in range(0, ncol, blk):
        nb = min(blk, ncol - c0)
        part = atm_to_device(S.make_atmosphere(nb, nlay, seed=shard.rank_seed(args.seed + 5, rank) + c0, clouds=True),
                             torch.float32, dev)
        if atm is None:
            atm = {k: (torch.empty(v.shape[:-1] + (ncol,), dtype=v.dtype, device=dev) if v.dim() and
                       v.shape[-1] == nb and k not in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif")
                       else None) for k, v in part.items() if k != "gases"}
            for k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif"):
                atm[k] = torch.empty((ncol,) + part[k].shape[1:], dtype=torch.float32, device=dev)
            atm["gases"] = {k: (torch.empty(v.shape[:-1] + (ncol,), dtype=v.dtype, device=dev) if v.numel() > 1
                                else v.clone()) for k, v in part["gases"].items()}
        for k, v in part.items():
            if k == "gases":
                for g, t in v.items():
                    if t.numel() > 1:
                        atm["gases"][g][..., c0:c0 + nb].copy_(t)
            elif k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif"):
                atm[k][c0:c0 + nb].copy_(v)
            elif atm.get(k) is not None:
                atm[k][..., c0:c0 + nb].copy_(v)
        del part
    nlev = nlay + 1
    gen = torch.Generator(device=dev).manual_seed(args.seed)
    sd = {k: torch.randn(shape, generator=gen, device=dev) for k, shape in
          (("up", (nlev, ncol)), ("dn", (nlev, ncol)), ("dir", (nlev, ncol)), ("hr", (nlay, ncol)))}

    def run(ev=None):
        # one launch per domain: fluxes and gradients
        if ev is not None:
            ev[0].record(stream)
        res_lw = adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"], with_fluxes=True)
        if ev is not None:
            ev[1].record(stream)
        res_sw = adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"], with_fluxes=True)
        if ev is not None:
            ev[2].record(stream)
        return res_lw[0], res_sw[0]

    run()
    torch.cuda.synchronize()
    evs = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(args.deep_steps)]
    for e in evs:
        flush.zero_()
        f_lw, f_sw = run(e)
    torch.cuda.synchronize()
    parts = [float(np.mean([e[q].elapsed_time(e[q + 1]) for e in evs])) for q in range(2)]
    tot = shard.max_over_ranks(float(np.sum(parts)), dist if world > 1 else None, dev)
    # FP64 forward of this build on one 8192-column block of the same atmosphere
    nb = min(8192, ncol)
    sub = {k: (v[..., :nb] if k not in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif") else v[:nb])
           for k, v in atm.items() if k != "gases" and v is not None}
    sub = {k: v.double().contiguous() for k, v in sub.items()}
    sub["gases"] = {k: (v[..., :nb] if v.numel() > 1 else v).double().contiguous() for k, v in atm["gases"].items()}
    solver.solve_lw(sub)
    solver.solve_sw(sub)
    torch.cuda.synchronize()
    e64 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2)]
    for a, b in e64:
        flush.zero_()
        a.record(stream)
        solver.solve_lw(sub)
        solver.solve_sw(sub)
        b.record(stream)
    torch.cuda.synchronize()
    ms64 = float(np.mean([a.elapsed_time(b) for a, b in e64]))
    r_lw, r_sw = solver.solve_lw(sub), solver.solve_sw(sub)
    ferr = max(float((f[k][:, :nb].double() - r[k]).abs().max()) for f, r in ((f_lw, r_lw), (f_sw, r_sw))
               for k in ("flux_up", "flux_dn", "flux_net"))
    herr = max(float((f["heating_rate"][:, :nb].double() - r["heating_rate"]).abs().max())
               for f, r in ((f_lw, r_lw), (f_sw, r_sw)))
    solver._bufs = {k: v for k, v in solver._bufs.items() if k[0][2] != torch.float64}
    fwd_adj = ncol * world / (tot * 1e-3)
    fp64 = nb / (ms64 * 1e-3)
    out = {"workload": f"all-sky LW+SW forward + adjoint, ncol={ncol} per GPU, nlay={nlay}",
           "forward_adjoint": {"value": fwd_adj, "unit": "columns/s", "ms_per_step": tot, "steps": args.deep_steps,
                               "kernel_ms": {"lw_adjoint_kernel (with fluxes)": round(parts[0], 3),
                                             "sw_adjoint_kernel (with fluxes)": round(parts[1], 3)}},
           "fp64_forward_blocked": {"value": fp64, "unit": "columns/s", "block_ncol": nb, "ms_per_block": ms64},
           "ratio_fwd_adj_over_fp64": fwd_adj / (fp64 * world),
           "fp32_max_flux_err_w_m2": ferr, "fp32_max_heating_rate_err_k_day": herr}
    del atm, sd, sub, f_lw, f_sw
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference-gpu-child":
        return run_reference_gpu_child(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from rrtmgp_b200 import shard
    from rrtmgp_b200 import synthetic as S
    from rrtmgp_b200.solver import Fused_solver, Radiation_solver, atm_to_device

    tables = {"lw": S.make_kdist("lw"), "sw": S.make_kdist("sw"),
              "cloud_lw": S.make_cloud_luts("lw"), "cloud_sw": S.make_cloud_luts("sw")}
    atm_np = S.make_atmosphere(args.ncol, args.nlay, seed=shard.rank_seed(args.seed, rank), clouds=True)
    solver = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
    fused = Fused_solver(solver)
    run_lw = fused.solve_lw if args.path == "fused" else solver.solve_lw
    run_sw = fused.solve_sw if args.path == "fused" else solver.solve_sw
    atm = atm_to_device(atm_np, torch.float32, dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    stages = {}

    def evpair():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step(timed_events=None):
        if timed_events is None:
            run_lw(atm)
            run_sw(atm)
            return
        a, m, b = timed_events
        a.record(stream)
        run_lw(atm)
        m.record(stream)
        run_sw(atm)
        b.record(stream)

    # Per-stage timing pass (same kernels, events around each stage) for the roofline.
    def staged_breakdown(reps):
        import ctypes as C
        from rrtmgp_b200 import _abi, api
        lib = _abi.load()
        res = {}
        b_lw = solver._buffers((args.ncol, args.nlay, torch.float32), atm["play"], args.ncol, args.nlay, "lw")
        ncol, nlay = args.ncol, args.nlay
        P = api._ptr
        s = api._stream()
        arr, keep = api.Gas_optics_rrtmgp._gases(atm["gases"], ncol, nlay, atm["play"])

        def t_gas_lw():
            lib.rrtmgp_b200_gas_optics_lw_f32(solver.klw.handle, ncol, nlay, P(atm["play"]), P(atm["plev"]),
                                              P(atm["tlay"]), P(atm["tsfc"]), P(atm["tlev"]), None, arr,
                                              len(atm["gases"]), P(b_lw["tau"]), P(b_lw["lay_src"]),
                                              P(b_lw["lev_src_inc"]), P(b_lw["lev_src_dec"]), P(b_lw["sfc_src"]),
                                              P(b_lw["sfc_src_jac"]), s)

        def t_lw_solver():
            lib.rrtmgp_b200_rte_lw_f32(solver.klw.bands.handle, ncol, nlay, 1, P(b_lw["tau"]), P(b_lw["lay_src"]),
                                       P(b_lw["lev_src_inc"]), P(b_lw["lev_src_dec"]), P(b_lw["sfc_src"]),
                                       P(atm["emis_sfc"]), None, 1, P(b_lw["gpt_up"]), P(b_lw["gpt_dn"]), s)

        b_sw = solver._buffers((args.ncol, args.nlay, torch.float32), atm["play"], args.ncol, args.nlay, "sw")

        def t_gas_sw():
            lib.rrtmgp_b200_gas_optics_sw_f32(solver.ksw.handle, ncol, nlay, P(atm["play"]), P(atm["plev"]),
                                              P(atm["tlay"]), None, arr, len(atm["gases"]), P(b_sw["tau"]),
                                              P(b_sw["ssa"]), P(b_sw["g"]), P(b_sw["toa_src"]), s)

        def t_sw_solver():
            lib.rrtmgp_b200_rte_sw_f32(solver.ksw.bands.handle, ncol, nlay, 1, P(b_sw["tau"]), P(b_sw["ssa"]),
                                       P(b_sw["g"]), P(atm["mu0"]), P(b_sw["toa_src"]), P(atm["sfc_alb_dir"]),
                                       P(atm["sfc_alb_dif"]), None, P(b_sw["gpt_up"]), P(b_sw["gpt_dn"]),
                                       P(b_sw["gpt_dir"]), C.c_void_p(b_sw["ws"].data_ptr()),
                                       C.c_size_t(b_sw["ws"].numel()), s)

        def t_bb_lw():
            lib.rrtmgp_b200_fluxes_broadband_f32(ncol, nlay + 1, 256, P(b_lw["gpt_up"]), P(b_lw["gpt_dn"]), None,
                                                 P(b_lw["flux_up"]), P(b_lw["flux_dn"]), None, P(b_lw["flux_net"]), s)

        for name, fn in (("gas_optics_lw", t_gas_lw), ("lw_solver", t_lw_solver), ("gas_optics_sw", t_gas_sw),
                         ("sw_solver", t_sw_solver), ("broadband_lw", t_bb_lw)):
            # untimed launches first: on the fused path these kernels have not run yet in this
            # process, and a first launch carries their one-time set-up (module load, shared-memory
            # opt-in, tensor-map encoder lookup)
            for _ in range(2):
                fn()
            torch.cuda.synchronize()
            ms = []
            for _ in range(reps):
                flush.zero_()
                e0, e1 = evpair()
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            res[name] = float(np.mean(ms))
        return res

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    evs = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()          # L2 flush between timed steps (outside the events)
        step(evs[i])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, m, b in evs]
    lw_ms = float(np.mean([a.elapsed_time(m) for a, m, b in evs]))
    sw_ms = float(np.mean([m.elapsed_time(b) for a, m, b in evs]))
    total_ms = float(np.sum(step_ms))
    total_ms = shard.max_over_ranks(total_ms, dist if world > 1 else None, dev)
    ms_per_step = total_ms / args.steps
    value = shard.weak_scaling_rate(args.ncol, world, args.steps, total_ms)

    # Per-kernel durations and roofline of the dominant kernel.
    traffic = ncu_traffic()
    hbm_peak, peak_kind = measured_peaks()
    if args.path == "fused":
        # One kernel per solve: the events around each solve inside the timed steps time it.
        breakdown = {"lw_forward_kernel": lw_ms, "sw_forward_kernel": sw_ms}
        dom = max(breakdown, key=breakdown.get)
        fpc = fused_flops_per_column(args.nlay)
        bpc = fused_bytes_per_column(args.nlay)
        peak_tf = fp32_peak(torch, dev, stream)
        achieved = fpc[dom] * args.ncol / (breakdown[dom] * 1e-3) / 1e12
        hbm_ach = bpc[dom] * args.ncol / (breakdown[dom] * 1e-3) / 1e9
        roofline = {"bound": "fp32", "kernel": dom, "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                    "frac": achieved / peak_tf,
                    "peak_source": "measured: FP32 FMA probe (rrtmgp_b200_fp32_fma_probe) on this GPU",
                    "traffic": traffic[dom] * args.ncol if dom in traffic else None,
                    "algorithmic_flops": fpc[dom] * args.ncol, "algorithmic_bytes": bpc[dom] * args.ncol,
                    "hbm": {"achieved": hbm_ach, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_ach / hbm_peak,
                            "peak_source": peak_kind},
                    "kernel_ms": {k: round(v, 4) for k, v in breakdown.items()}}
    else:
        breakdown = staged_breakdown(10)
        bpc = bytes_per_column(args.nlay)
        dom = max(breakdown, key=breakdown.get)
        achieved = bpc[dom] * args.ncol / (breakdown[dom] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": achieved / hbm_peak, "peak_source": peak_kind,
                    "traffic": traffic[dom] * args.ncol if dom in traffic else None,
                    "algorithmic_bytes": bpc[dom] * args.ncol,
                    "kernel_ms": {k: round(v, 4) for k, v in breakdown.items()}}

    # Per-stage kernels of the class API (FP32), each against its HBM roofline.
    staged_kernels = None
    if args.path == "fused" and rank == 0:
        sk = staged_breakdown(10)
        bpc_s = bytes_per_column(args.nlay)
        staged_kernels = {}
        for k, ms in sk.items():
            gbs = bpc_s[k] * args.ncol / (ms * 1e-3) / 1e9
            staged_kernels[k] = {"ms": round(ms, 4), "algorithmic_bytes": bpc_s[k] * args.ncol,
                                 "achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm_peak, 4)}

    # End to end through the public API with host buffers (pinned), copies in the timed region.
    in_keys = ["play", "plev", "tlay", "tlev", "tsfc", "lwp", "iwp", "rel", "rei", "mu0", "emis_sfc",
               "sfc_alb_dir", "sfc_alb_dif"]
    host_in = {k: atm[k].cpu().pin_memory() for k in in_keys}
    host_gas = {k: v.cpu().pin_memory() for k, v in atm["gases"].items()}
    out_lw = run_lw(atm)
    out_sw = run_sw(atm)
    host_out = {("lw", k): v.cpu().pin_memory() for k, v in out_lw.items()}
    host_out.update({("sw", k): v.cpu().pin_memory() for k, v in out_sw.items()})
    h2d = sum(v.numel() * v.element_size() for v in host_in.values()) + \
        sum(v.numel() * v.element_size() for v in host_gas.values())
    d2h = sum(v.numel() * v.element_size() for v in host_out.values())

    def e2e_step():
        for k in in_keys:
            atm[k].copy_(host_in[k], non_blocking=True)
        for k in host_gas:
            atm["gases"][k].copy_(host_gas[k], non_blocking=True)
        o1 = run_lw(atm)
        o2 = run_sw(atm)
        for k, v in o1.items():
            host_out[("lw", k)].copy_(v, non_blocking=True)
        for k, v in o2.items():
            host_out[("sw", k)].copy_(v, non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ee = [evpair() for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ee[i][0].record(stream)
        e2e_step()
        ee[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = float(np.sum([a.elapsed_time(b) for a, b in ee]))
    e2e_value = shard.weak_scaling_rate(args.ncol, world, args.steps,
                                        shard.max_over_ranks(e2e_ms, dist if world > 1 else None, dev))
    e2e_serial = e2e_value

    # The same, pipelined: the columns in blocks on two streams, so that the host copies of one
    # block overlap the kernels of the other.  Each block has its own pinned host buffers and
    # device arrays (a caller with one large host array would stage it in blocks the same way);
    # blocks on one stream reuse its solver's output buffers in stream order.
    # 8 blocks at 8192 columns (1024 per launch): the first block's input copy and the last
    # block's output copy, the only ones not overlapped, are 1/8 of a step's copies
    nblk = 8 if args.ncol >= 8 * 1024 else (4 if args.ncol >= 4 * 256 else 1)
    edges = [int(x) for x in np.linspace(0, args.ncol, nblk + 1)]

    def col_block(t, a, b):
        if t.dim() == 2 and t.shape[1] == args.ncol:
            return t[:, a:b]
        if t.dim() >= 1 and t.shape[0] == args.ncol:
            return t[a:b]
        return t

    if args.path == "fused":
        slots = [(fused.solve_lw, fused.solve_sw)]
        f2 = Fused_solver(solver)
        slots.append((f2.solve_lw, f2.solve_sw))
    else:
        s2 = Radiation_solver(tables["lw"], tables["sw"], tables["cloud_lw"], tables["cloud_sw"], S.ATM_GASES)
        slots = [(solver.solve_lw, solver.solve_sw), (s2.solve_lw, s2.solve_sw)]
    streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
    blocks = []
    for bi in range(nblk):
        a, b = edges[bi], edges[bi + 1]
        hin = {k: col_block(host_in[k], a, b).contiguous().pin_memory() for k in in_keys}
        hgas = {k: col_block(v, a, b).contiguous().pin_memory() for k, v in host_gas.items()}
        din = {k: v.to(dev) for k, v in hin.items()}
        din["gases"] = {k: v.to(dev) for k, v in hgas.items()}
        lw_o = slots[bi % 2][0](din)
        sw_o = slots[bi % 2][1](din)
        hout = {("lw", k): v.cpu().pin_memory() for k, v in lw_o.items()}
        hout.update({("sw", k): v.cpu().pin_memory() for k, v in sw_o.items()})
        blocks.append((hin, hgas, din, hout))
    torch.cuda.synchronize()

    def e2e_pipelined_step():
        start = torch.cuda.Event()
        start.record(stream)
        for bi, (hin, hgas, din, hout) in enumerate(blocks):
            st = streams[bi % 2]
            st.wait_event(start)
            with torch.cuda.stream(st):
                for k in in_keys:
                    din[k].copy_(hin[k], non_blocking=True)
                for k in hgas:
                    din["gases"][k].copy_(hgas[k], non_blocking=True)
                o1 = slots[bi % 2][0](din)
                o2 = slots[bi % 2][1](din)
                for k, v in o1.items():
                    hout[("lw", k)].copy_(v, non_blocking=True)
                for k, v in o2.items():
                    hout[("sw", k)].copy_(v, non_blocking=True)
        for st in streams:
            done = torch.cuda.Event()
            done.record(st)
            stream.wait_event(done)

    for _ in range(2):
        e2e_pipelined_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ep = [evpair() for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ep[i][0].record(stream)
        e2e_pipelined_step()
        ep[i][1].record(stream)
    torch.cuda.synchronize()
    ep_ms = float(np.sum([a.elapsed_time(b) for a, b in ep]))
    e2e_value = shard.weak_scaling_rate(args.ncol, world, args.steps,
                                        shard.max_over_ranks(ep_ms, dist if world > 1 else None, dev))
    # outputs of the pipelined blocks equal the one-launch outputs
    e2e_check = max(float((hout[("sw", "flux_dn")].double() - out_sw["flux_dn"].cpu().double()[:, edges[bi]:edges[bi + 1]]).abs().max())
                    for bi, (_, _, _, hout) in enumerate(blocks))

    # FP32 forward + hand-written adjoint (LW and SW), seeded on every output: the path the
    # FP32 target is stated on.  Same columns, L2 flushed between steps, events per kernel.
    fwd_adj = None
    if args.path == "fused" and not args.no_adjoint:
        from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
        nlev = args.nlay + 1
        gen = torch.Generator(device=dev).manual_seed(args.seed)
        sd = {k: torch.randn(shape, generator=gen, device=dev) for k, shape in
              (("up", (nlev, args.ncol)), ("dn", (nlev, args.ncol)), ("dir", (nlev, args.ncol)),
               ("hr", (args.nlay, args.ncol)))}

        def fa_step(e=None):
            # one launch per domain: fluxes and gradients (rrtmgp_b200_forward_adjoint_*_f32)
            if e is not None:
                e[0].record(stream)
            adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"], with_fluxes=True)
            if e is not None:
                e[1].record(stream)
            adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"], with_fluxes=True)
            if e is not None:
                e[2].record(stream)

        def separate_step(e):
            e[0].record(stream)
            run_lw(atm)
            e[1].record(stream)
            adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"])
            e[2].record(stream)
            run_sw(atm)
            e[3].record(stream)
            adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"])
            e[4].record(stream)

        for _ in range(2):
            fa_step()
        torch.cuda.synchronize()
        nrep = max(2, args.steps // 5)
        ev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(nrep)]
        for i in range(nrep):
            flush.zero_()
            fa_step(ev[i])
        torch.cuda.synchronize()
        parts = [float(np.mean([e[q].elapsed_time(e[q + 1]) for e in ev])) for q in range(2)]
        tot = shard.max_over_ranks(float(np.sum(parts)), dist if world > 1 else None, dev)
        # the same work as separate forward and adjoint launches (breakdown)
        ev2 = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(5)) for _ in range(2)]
        for e in ev2:
            flush.zero_()
            separate_step(e)
        torch.cuda.synchronize()
        sep = [float(np.mean([e[q].elapsed_time(e[q + 1]) for e in ev2])) for q in range(4)]
        fwd_adj = {"value": shard.weak_scaling_rate(args.ncol, world, 1, tot), "unit": "columns/s",
                   "ms_per_step": tot, "steps": nrep, "gpu_launches_per_step": 2,
                   "kernel_ms": {"lw_adjoint_kernel (with fluxes)": round(parts[0], 4),
                                 "sw_adjoint_kernel (with fluxes)": round(parts[1], 4)},
                   "separate_launches_ms": {"lw_forward_kernel": round(sep[0], 4),
                                            "lw_adjoint_kernel": round(sep[1], 4),
                                            "sw_forward_kernel": round(sep[2], 4),
                                            "sw_adjoint_kernel": round(sep[3], 4), "total": round(sum(sep), 4)},
                   "gradients": "flux/heating-rate seeds -> tlay, tlev, tsfc, h2o, o3, lwp, iwp, rel, rei (LW); "
                                "tlay, h2o, o3, lwp, iwp, rel, rei, surface albedos (SW); fluxes and heating "
                                "rates from the same launches"}

    # Plain FP64 GPU forward of the same build (the denominator of the FP32 target).
    fp64 = None
    if not args.no_fp64:
        atm64 = atm_to_device(atm_np, torch.float64, dev)
        solver.solve_lw(atm64)
        solver.solve_sw(atm64)
        torch.cuda.synchronize()
        nrep = max(2, args.steps // 3)
        e64 = [evpair() for _ in range(nrep)]
        for i in range(nrep):
            flush.zero_()
            e64[i][0].record(stream)
            solver.solve_lw(atm64)
            solver.solve_sw(atm64)
            e64[i][1].record(stream)
        torch.cuda.synchronize()
        ms64 = float(np.mean([a.elapsed_time(b) for a, b in e64]))
        # Accuracy of the timed FP32 path against this FP64 forward on the bench workload.
        r_lw, r_sw = solver.solve_lw(atm64), solver.solve_sw(atm64)
        f_lw, f_sw = run_lw(atm), run_sw(atm)
        ferr = max(float((f[k].double() - r[k]).abs().max()) for f, r in ((f_lw, r_lw), (f_sw, r_sw))
                   for k in ("flux_up", "flux_dn", "flux_net"))
        herr = max(float((f["heating_rate"].double() - r["heating_rate"]).abs().max())
                   for f, r in ((f_lw, r_lw), (f_sw, r_sw)))
        fp64 = {"value": args.ncol / (ms64 * 1e-3), "unit": "columns/s", "ms_per_step": ms64,
                "fp32_max_flux_err_w_m2": ferr, "fp32_max_heating_rate_err_k_day": herr}
        if fwd_adj is not None:
            # the fluxes of the forward + adjoint launches against the same FP64 forward
            from rrtmgp_b200.autodiff import adjoint_lw, adjoint_sw
            a_lw = adjoint_lw(fused, atm, sd["up"], sd["dn"], sd["hr"], with_fluxes=True)[0]
            a_sw = adjoint_sw(fused, atm, sd["up"], sd["dn"], sd["dir"], sd["hr"], with_fluxes=True)[0]
            fwd_adj["fp32_max_flux_err_w_m2"] = max(float((f[k].double() - r[k]).abs().max())
                                                    for f, r in ((a_lw, r_lw), (a_sw, r_sw))
                                                    for k in ("flux_up", "flux_dn", "flux_net"))
            fwd_adj["fp32_max_heating_rate_err_k_day"] = max(
                float((f["heating_rate"].double() - r["heating_rate"]).abs().max()) for f, r in ((a_lw, r_lw), (a_sw, r_sw)))
        del atm64
        solver._bufs = {k: v for k, v in solver._bufs.items() if k[0][2] != torch.float64}

    # Aerosol optics (the SW band LUT by relative humidity): one launch over the bench columns;
    # HBM-bound streaming (13 (ncol, nlay) fields in, tau/ssa/g per band out).
    aer_line = None
    if args.path == "fused":
        from rrtmgp_b200 import api
        aer_np, rh_np = S.make_aerosols(atm_np["play"], seed=args.seed + 9)
        ao = api.Aerosol_optics(S.make_aerosol_luts())
        aer_t = {k: torch.as_tensor(v, dtype=torch.float32, device=dev) for k, v in aer_np.items()}
        rh_t = torch.as_tensor(rh_np, dtype=torch.float32, device=dev)
        for _ in range(3):
            ao.aerosol_optics(aer_t, rh_t, atm["plev"])
        torch.cuda.synchronize()
        ev = [evpair() for _ in range(5)]
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            ao.aerosol_optics(aer_t, rh_t, atm["plev"])
            b.record(stream)
        torch.cuda.synchronize()
        ms = float(np.median([a.elapsed_time(b) for a, b in ev]))
        nb = ao.nband
        nbytes = 4 * args.ncol * (13 * args.nlay + 1 + 3 * nb * args.nlay)
        gbs = nbytes / (ms * 1e-3) / 1e9
        aer_line = {"workload": f"aerosol optics, 11 species, ncol={args.ncol}, nlay={args.nlay}, {nb} bands",
                    "ms": ms, "columns_per_s": args.ncol / (ms * 1e-3),
                    "roofline": {"bound": "hbm", "algorithmic_bytes": nbytes, "achieved": gbs, "peak": hbm_peak,
                                 "unit": "GB/s", "frac": gbs / hbm_peak, "peak_source": peak_kind}}
        del aer_t, rh_t

    deep = None
    if args.path == "fused" and args.deep_ncol > 0 and not args.no_adjoint:
        deep = deep_bench(args, solver, fused, dev, stream, flush, rank, world, dist)

    batched = None
    if args.path == "fused" and args.batched_grids > 0:
        batched = batched_bench(args, solver, dev, stream, flush, rank, world, dist)

    # staged: LW gas, cloud, add_to, rte, reduce, heating; SW the same + spread, delta.
    launches_per_step = 2 if args.path == "fused" else 6 + 8
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, tables, args.cpu_seconds)

    if rank == 0:
        # The metric's own quantity: FP32 forward + adjoint columns/s over the plain FP64 GPU
        # forward of this build, with the FP32 errors against that FP64 forward.
        headline = None
        if fp64 is not None and fwd_adj is not None:
            headline = {"fwd_adj_over_fp64": fwd_adj["value"] / (fp64["value"] * world),
                        "fp32_forward_over_fp64": value / (fp64["value"] * world),
                        "fp32_fwd_adj_columns_per_s": fwd_adj["value"],
                        "fp64_forward_columns_per_s": fp64["value"] * world,
                        "fp32_max_flux_err_w_m2": fwd_adj.get("fp32_max_flux_err_w_m2"),
                        "fp32_max_heating_rate_err_k_day": fwd_adj.get("fp32_max_heating_rate_err_k_day"),
                        "target": ">= 3x the plain FP64 forward, errors <= 0.05 W/m2 and 0.01 K/day"}
        line = {
            "metric": METRIC, "value": value, "unit": "columns/s", "headline": headline,
            "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"all-sky LW+SW forward (gas+cloud optics, rte_lw, rte_sw, broadband fluxes, "
                                   f"heating rates), ncol={args.ncol} per GPU, nlay={args.nlay}, 256 LW / 224 SW "
                                   f"g-points, synthetic tables",
                       "ncol": args.ncol, "nlay": args.nlay, "path": args.path,
                       "l2": "flushed between timed steps (256 MiB write outside the events)",
                       "parallelism": f"columns sharded over {world} GPU(s), no exchange"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "columns/s", "h2d_bytes_per_step": h2d * world,
                    "d2h_bytes_per_step": d2h * world,
                    "pipeline": f"{nblk} column blocks on 2 streams: host copies of a block overlap the "
                                f"kernels of another",
                    "serial_value": e2e_serial, "max_diff_vs_one_launch_w_m2": e2e_check},
            "gpu_launches": launches_per_step * args.steps,
            "fp64_forward": fp64,
            "forward_adjoint": fwd_adj,
            "deep_forward_adjoint": deep,
            "clocks": clocks,
            "aerosol_optics": aer_line,
            "staged_kernels": staged_kernels,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
