"""Multi-GPU sharding of a simulation batch.

The reference runs one process per GPU over disjoint row ranges of MX_0 /
c_matrix (the `offset` argument, kernel.cu:91-95).  Here every rank takes a
contiguous range and passes its first global row as `sim_base`, so the
Philox streams -- and therefore every trajectory -- are those of one large
single-process run.  Dynamics need no collective.  The fitness mode needs
ensemble statistics over all replicates: per (instant, species) the sum and
the sum of squares, one all-reduce of 2 x ns x S doubles.
"""
from __future__ import annotations

import numpy as np


def shard_range(n_total: int, rank: int, world: int):
    """(offset, count) of rank's contiguous share; the first n_total % world
    ranks take one extra row."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n_total, world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def local_stats(samples) -> np.ndarray:
    """[2][ns][S] float64: sum and sum of squares over the simulations of
    samples [n][ns][S]."""
    x = np.asarray(samples, dtype=np.float64)
    return np.stack([x.sum(0), (x * x).sum(0)])


def ensemble_stats(samples, n_total: int, dist=None, device="cpu"):
    """Mean and unbiased variance per (instant, species) over all ranks."""
    st = local_stats(samples)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        import torch
        t = torch.as_tensor(st, device=device)
        dist.all_reduce(t)
        st = t.cpu().numpy()
    mean = st[0] / n_total
    var = (st[1] - n_total * mean * mean) / max(1, n_total - 1)
    return mean, var


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The step time of a multi-rank run: the slowest rank's."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
