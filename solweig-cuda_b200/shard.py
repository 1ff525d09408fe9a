"""Sharding of independent work units over ranks (one process per GPU).

Days are independent because the thermal state resets every calendar day
(``src/series.py:425-436``) and tiles are independent given a halo
(``src/tiling.py:29-42``), so ranks split them without any data-path
collective; the only collectives are the timing reduction (max over ranks)
and barriers.
"""
from __future__ import annotations

__all__ = ["split", "max_over_ranks"]


def split(units, rank, world):
    """Contiguous, balanced share of ``units`` (a sequence) for ``rank`` of ``world``."""
    n = len(units)
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return units[start:stop]


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
