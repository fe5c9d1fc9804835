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
import pytest
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
