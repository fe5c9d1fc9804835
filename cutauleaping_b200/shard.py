"""Multi-GPU sharding of a simulation batch.

The reference runs one process per GPU over disjoint row ranges of MX_0 /
c_matrix (the `offset` argument, kernel.cu:91-95).  Here every rank takes a
contiguous range and passes its first global row as `sim_base`, so the
Philox streams -- and therefore every trajectory -- are those of one large
single-process run.  Dynamics need no collective.  The fitness mode needs
ensemble statistics over all replicates: per (instant, species) each rank's
count, mean and sum of squared deviations, one all-gather of 3 x ns x S
doubles per rank, merged by Chan et al.'s pairwise update.  Data-parallel
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
    """[3][ns][S] float64 over the simulations of samples [n][ns][S]: the
    count n, the mean and M2 = the sum of squared deviations from the mean.
    Deviations from the local mean keep M2 exact to rounding where a raw sum
    of squares (counts near 1e6 over tens of thousands of simulations passes
    2^53) would lose its digits to cancellation."""
    x = np.asarray(samples, dtype=np.float64)
    n = x.shape[0]
    if n == 0:
        z = np.zeros(x.shape[1:])
        return np.stack([z, z, z])
    mean = x.mean(0)
    d = x - mean
    return np.stack([np.full(mean.shape, float(n)), mean, (d * d).sum(0)])


def merge_stats(parts) -> np.ndarray:
    """Chan, Golub and LeVeque's pairwise update of (count, mean, M2),
    applied to the parts in the order given (every rank merges the same
    list, so every rank gets the same bits)."""
    n, mean, m2 = (np.array(v, dtype=np.float64) for v in parts[0])
    for p in parts[1:]:
        nb, mb, m2b = p
        tot = n + nb
        safe = np.where(tot > 0, tot, 1.0)
        delta = mb - mean
        mean = np.where(tot > 0, mean + delta * (nb / safe), mean)
        m2 = m2 + m2b + delta * delta * (n * nb / safe)
        n = tot
    return np.stack([n, mean, m2])


def ensemble_stats(samples, n_total: int, dist=None, device="cpu"):
    """Mean and unbiased variance per (instant, species) over all ranks: one
    all-gather of every rank's (count, mean, M2), merged in rank order."""
    st = local_stats(samples)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        import torch
        t = torch.as_tensor(st, device=device)
        parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
        dist.all_gather(parts, t)
        st = merge_stats([p.cpu().numpy() for p in parts])
    if int(round(float(st[0].flat[0]))) != n_total:
        raise ValueError(f"the ranks hold {int(st[0].flat[0])} simulations, expected {n_total}")
    return st[1], st[2] / max(1, n_total - 1)


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
