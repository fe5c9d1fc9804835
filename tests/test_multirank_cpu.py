"""Multi-rank host logic on CPU (gloo, world size 2).

Each rank simulates its shard of a batch with the CPU oracle (standing in
for one GPU: the device sweep is bit-identical to it, tests/test_gpu_parity),
using the shard's first global row as sim_base; the all-reduced ensemble
statistics must equal those of one process simulating the whole batch, and the
max-over-ranks timing must return the slowest rank's value.
"""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from cutauleaping_b200 import inputs, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from tests.netutil import oracle_model
        net = inputs.schlogl(96, samples=20, t_end=1.0)
        off, cnt = shard.shard_range(net.n, rank, world)
        m = oracle_model(net, seed=9)
        out, _ = m.run(net.X0[off:off + cnt], net.c[off:off + cnt].astype(np.float32), sim_base=off, threads=2)
        mean, var = shard.ensemble_stats(out, net.n, dist)
        slow = shard.max_over_ranks(float(rank + 1) * 10.0, dist)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), mean=mean, var=var, slow=slow, off=off, cnt=cnt,
                 out=out)
    finally:
        dist.destroy_process_group()


def test_merged_stats_keep_digits_at_large_counts():
    """Counts near 1e6 over many simulations: the sum of squares passes 2^53,
    so a variance from raw sums loses its digits; the pairwise merge of
    per-part (count, mean, M2) keeps them."""
    rng = np.random.default_rng(0)
    x = (1_000_000 + rng.integers(-3, 4, size=(65536, 2, 3))).astype(np.float64)
    exact_var = x.var(axis=0, ddof=1)
    parts = [shard.local_stats(x[a:b]) for a, b in ((0, 1000), (1000, 40000), (40000, 65536))]
    st = shard.merge_stats(parts)
    assert np.array_equal(st[0], np.full((2, 3), 65536.0))
    assert np.allclose(st[1], x.mean(0), rtol=1e-15, atol=0)
    assert np.allclose(st[2] / 65535, exact_var, rtol=1e-9, atol=0)
    raw = ((x * x).sum(0) - 65536 * x.mean(0) ** 2) / 65535
    assert not np.allclose(raw, exact_var, rtol=1e-3, atol=0)   # what the merge avoids


def test_shard_ranges_cover_the_batch():
    for n in (1, 7, 96, 1001):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_range(n, r, world) for r in range(world)]
            assert sum(c for _, c in parts) == n
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))


def test_two_ranks_reproduce_single_process(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(2))
    from tests.netutil import oracle_model
    net = inputs.schlogl(96, samples=20, t_end=1.0)
    full, _ = oracle_model(net, seed=9).run(net.X0, net.c.astype(np.float32), threads=2)
    # the shards are exactly the rows of the single run
    assert np.array_equal(np.concatenate([r0["out"], r1["out"]]), full)
    mean, var = shard.ensemble_stats(full, net.n)
    for r in (r0, r1):
        assert np.allclose(r["mean"], mean, rtol=0, atol=1e-9)
        assert np.allclose(r["var"], var, rtol=1e-12, atol=1e-9)
        assert float(r["slow"]) == 20.0


def _dp_worker(rank, world, port, out_dir):
    """Data-parallel training step on CPU: each rank takes its shard of one
    batch, the gradients are averaged with shard.allreduce_mean, and every
    rank applies the same update."""
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the averaging itself, on tensors of several shapes
        a = torch.full((3, 4), float(rank + 1))
        b = torch.arange(5, dtype=torch.float32) * (rank + 1)
        shard.allreduce_mean([a, b], dist)
        # rank 0's scaling wins
        sc = torch.tensor([float(rank) + 0.5, 2.0 * rank])
        shard.broadcast_([sc], dist)
        # a linear least-squares model trained by gradient descent
        g = torch.Generator().manual_seed(4)
        X = torch.randn(64, 5, generator=g, dtype=torch.float64)
        y = X @ torch.tensor([1.0, -2.0, 0.5, 3.0, -1.0], dtype=torch.float64) + 0.1
        off, cnt = shard.shard_range(64, rank, world)
        w = torch.zeros(5, dtype=torch.float64, requires_grad=True)
        c = torch.zeros(1, dtype=torch.float64, requires_grad=True)
        for _ in range(20):
            loss = ((X[off:off + cnt] @ w + c - y[off:off + cnt]) ** 2).mean()
            gw, gc = torch.autograd.grad(loss, [w, c])
            gw, gc = gw.clone(), gc.clone()
            shard.allreduce_mean([gw, gc], dist)
            with torch.no_grad():
                w -= 0.1 * gw
                c -= 0.1 * gc
        np.savez(os.path.join(out_dir, f"dp{rank}.npz"), a=a.numpy(), b=b.numpy(), sc=sc.numpy(),
                 w=w.detach().numpy(), c=c.detach().numpy())
    finally:
        dist.destroy_process_group()


def test_data_parallel_gradient_average(tmp_path):
    """Two ranks, each with half of the batch, take the same steps as one
    process with the whole batch (equal shards: the mean of the shard means
    is the batch mean)."""
    import torch
    port = _free_port()
    mp.start_processes(_dp_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"dp{r}.npz") for r in range(2))
    for r in (r0, r1):
        assert np.array_equal(r["a"], np.full((3, 4), 1.5, np.float32))
        assert np.array_equal(r["b"], np.arange(5, dtype=np.float32) * 1.5)
        assert np.array_equal(r["sc"], np.array([0.5, 0.0], np.float32))
    assert np.array_equal(r0["w"], r1["w"]) and np.array_equal(r0["c"], r1["c"])
    g = torch.Generator().manual_seed(4)
    X = torch.randn(64, 5, generator=g, dtype=torch.float64)
    y = X @ torch.tensor([1.0, -2.0, 0.5, 3.0, -1.0], dtype=torch.float64) + 0.1
    w = torch.zeros(5, dtype=torch.float64, requires_grad=True)
    c = torch.zeros(1, dtype=torch.float64, requires_grad=True)
    for _ in range(20):
        loss = ((X @ w + c - y) ** 2).mean()
        gw, gc = torch.autograd.grad(loss, [w, c])
        with torch.no_grad():
            w -= 0.1 * gw
            c -= 0.1 * gc
    assert np.allclose(r0["w"], w.detach().numpy(), rtol=1e-12, atol=1e-12)
    assert np.allclose(r0["c"], c.detach().numpy(), rtol=1e-12, atol=1e-12)


def test_single_rank_helpers_are_no_ops():
    import torch
    t = torch.arange(4, dtype=torch.float32)
    assert shard.allreduce_mean([t], None)[0] is t and np.array_equal(t.numpy(), np.arange(4))
    assert not shard.multi_rank(None)
    assert shard.broadcast_([t], None)[0] is t
