"""Multi-GPU plumbing of the column path: columns are independent, so ranks own disjoint
column ranges and exchange nothing on the data path.  The only collective is the timing
reduction (max over ranks) and an optional gather of results on the host side.
"""
from __future__ import annotations


def column_range(ncol_total: int, rank: int, world: int):
    """Contiguous column range [start, stop) of `rank` when ncol_total columns are split over
    `world` ranks (strong scaling); ranges differ in length by at most one column."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(ncol_total, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def slice_columns(atm: dict, start: int, stop: int) -> dict:
    """Columns [start, stop) of an atmosphere in the binding's layout (numpy arrays or torch
    tensors): per-layer/level fields are (nlay[+1], ncol), per-column ones (ncol,) or
    (ncol, nband), gases either fields (nlay, ncol) or profiles/scalars, which every rank
    keeps whole.  Scalars (ncol, nlay, top_at_1) are adjusted or copied."""
    ncol = int(atm["ncol"]) if "ncol" in atm else int(atm["play"].shape[-1])
    if not 0 <= start <= stop <= ncol:
        raise ValueError(f"column range [{start}, {stop}) outside [0, {ncol})")
    out = {}
    for k, v in atm.items():
        if k == "gases":
            out[k] = {g: (a[:, start:stop] if a.ndim == 2 and a.shape[1] == ncol and a.shape[1] > 1 else a)
                      for g, a in v.items()}
        elif k == "ncol":
            out[k] = stop - start
        elif not hasattr(v, "ndim"):
            out[k] = v
        elif v.ndim == 1 and v.shape[0] == ncol:
            out[k] = v[start:stop]
        elif v.ndim == 2 and k in ("emis_sfc", "sfc_alb_dir", "sfc_alb_dif") and v.shape[0] == ncol:
            out[k] = v[start:stop]
        elif v.ndim == 2 and v.shape[1] == ncol:
            out[k] = v[:, start:stop]
        else:
            out[k] = v
    return out


def gather_columns(part: dict, dist=None) -> dict | None:
    """Host-side gather of per-rank results {name: array (..., ncol_rank)} (column last, numpy)
    into rank 0: returns the column-concatenated dict in rank order on rank 0, None on the
    others.  Without an initialised process group it returns `part`."""
    import numpy as np
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return part
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object({k: np.asarray(v) for k, v in part.items()}, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    return {k: np.concatenate([p[k] for p in parts], axis=-1) for k in part}


def rank_seed(seed: int, rank: int) -> int:
    """Seed of the synthetic atmosphere of `rank` (weak scaling: every rank owns its columns)."""
    return seed + rank


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank scalar (e.g. the timed milliseconds) over all ranks."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_rate(ncol_per_rank: int, world: int, steps: int, total_ms: float) -> float:
    """Whole-job columns/s when every rank processes ncol_per_rank columns per step."""
    return world * ncol_per_rank * steps / (total_ms * 1e-3)
