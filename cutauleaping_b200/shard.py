"""Multi-GPU sharding of a simulation batch.

The reference runs one process per GPU over disjoint row ranges of MX_0 /
c_matrix (the `offset` argument, kernel.cu:91-95).  Here every rank takes a
contiguous range and passes its first global row as `sim_base`, so the
Philox streams -- and therefore every trajectory -- are those of one large
single-process run.  Dynamics need no collective.  The fitness mode needs
ensemble statistics over all replicates: per (instant, species) the sum and
the sum of squares, one all-reduce of 2 x ns x S doubles.  Data-parallel
training of the surrogate averages its gradients over ranks: one all-reduce
of every weight and bias gradient packed into a single FP32 buffer
(about 0.2 M values for the 9 -> 256 x 4 -> 2S network).
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


def multi_rank(dist) -> bool:
    return dist is not None and dist.is_initialized() and dist.get_world_size() > 1


def allreduce_mean(tensors, dist=None):
    """Average a list of tensors over all ranks, in place, with one
    collective: the tensors are packed into one buffer of their common type
    (FP32 for the surrogate's gradients), all-reduced (sum), divided by the
    world size and unpacked.  With one rank (or no process group) the
    tensors are returned unchanged."""
    if not multi_rank(dist):
        return tensors
    import torch
    dtype = tensors[0].dtype
    for t in tensors[1:]:
        dtype = torch.promote_types(dtype, t.dtype)
    flat = torch.cat([t.reshape(-1).to(dtype) for t in tensors])
    dist.all_reduce(flat)
    flat /= dist.get_world_size()
    off = 0
    for t in tensors:
        k = t.numel()
        t.copy_(flat[off:off + k].view(t.shape))
        off += k
    return tensors


def broadcast_(tensors, dist=None, src: int = 0):
    """Overwrite each tensor with rank `src`'s copy (in place); a no-op with
    one rank."""
    if multi_rank(dist):
        for t in tensors:
            dist.broadcast(t, src=src)
    return tensors
