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
