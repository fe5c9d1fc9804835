"""GPU parity at the benchmark workloads' own sizes and launch plans.

The small-network parity tests (test_gpu_parity.py) cover every code path on
short runs.  These run each benchmark workload the way bench.py runs it --
the same network, batch, seed, t_end, sample instants and the library's launch
plan for the full batch -- and compare a spread subset of simulations bit for
bit against the CPU oracle (oracle/ctl_oracle.c, the restatement of
PreCalculations and EventualSSASteps, 2phase_n-tau-leaping.cu:1568-2273):
every sample and all seven per-simulation record fields.  Over full-length
trajectories (tens of thousands of steps) this exercises what short runs
cannot: step counters and Philox counters far from zero, attempt tags, long
chains of stored tree levels, and the multi-warp groups of the 512 x 1024
network.  One run goes through ctl_graph_create / ctl_graph_launch, the
bench's timed path.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs
from tests.netutil import oracle_model, same_info

pytestmark = pytest.mark.gpu

PLAN_FIELDS = ("group", "threads", "min_blocks", "sched", "ssa_budget", "dec_budget", "warp_sims")


def _plan_cfg(model, n_plan, seed, uniform, **over):
    """The library's launch plan for a batch of n_plan simulations, pinned
    as explicit settings (so a window of the batch runs the same plan).
    warp_sims > 0 selects the register-resident sweep (tiny networks); 0
    keeps the shared-memory sweep."""
    li = model.launch_info(n_plan, seed=seed, uniform_rates=uniform)
    kw = {f: getattr(li, f) for f in PLAN_FIELDS}
    kw.update(over)
    return li, kw


def _device(net, model, lo, hi, seed, kw, graph=False):
    """Rows [lo, hi) of the batch on device buffers (sim_base = lo); returns
    (samples, info) as numpy."""
    import torch
    n = hi - lo
    X0 = torch.from_numpy(np.ascontiguousarray(net.X0[lo:hi], np.int32)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(net.c[lo:hi], np.float32)).cuda()
    out = torch.full((n, model.ns, model.s_out), -1, dtype=torch.int32, device="cuda")
    info = torch.zeros((n, 40), dtype=torch.uint8, device="cuda")
    uniform = int(bool((net.c == net.c[0]).all()))
    cfg = ctl.run_cfg(seed=seed, sim_base=lo, uniform_rates=uniform, **kw)
    stream = torch.cuda.current_stream().cuda_stream
    if graph:
        g = model.graph(n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(), stream, cfg)
        g.launch(stream)
        torch.cuda.synchronize()
        out.fill_(-1)
        info.zero_()
        g.launch(stream)   # a replay reproduces the first launch's results
        torch.cuda.synchronize()
        del g
    else:
        model.run_device(n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(), stream, cfg)
        torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32), info.cpu().numpy().view(ctl.INFO_DTYPE).reshape(-1)


def _oracle_at(net, idx, seed):
    """The oracle's samples and records for the global simulations idx, each
    run on its own host thread (the C oracle releases the GIL)."""
    om = oracle_model(net, seed=seed)
    c32 = np.asarray(net.c, np.float32)

    def one(i):
        return om.run(net.X0[i:i + 1], c32[i:i + 1], sim_base=int(i), threads=1)
    with ThreadPoolExecutor(max(1, min(len(idx), 32))) as ex:
        res = list(ex.map(one, idx))
    return np.concatenate([r[0] for r in res]), np.concatenate([r[1] for r in res])


def _compare(net, out, info, lo, idx, seed, what):
    o_out, o_info = _oracle_at(net, idx, seed)
    rows = np.asarray(idx) - lo
    assert np.array_equal(out[rows], o_out), f"{what}: samples differ from the oracle"
    f = same_info(info[rows], o_info)
    assert f is None, f"{what}: record field {f} differs from the oracle"
    assert (info["status"] == ctl.SIM_OK).all(), f"{what}: a simulation ended early"
    return o_info


def test_config1_schlogl_full_batch_every_simulation():
    """Schlogl, 4,096 simulations, t_end 5, 100 samples: the whole batch
    compared (the slowest bistable simulations take about 14,000 steps)."""
    net = inputs.schlogl(4096)
    model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    li, kw = _plan_cfg(model, net.n, 1, 1)
    assert li.warp_sims > 0, "Schlogl's plan is the register-resident sweep"
    out, info = _device(net, model, 0, net.n, 1, kw)
    o_out, o_info = oracle_model(net, seed=1).run(net.X0, np.asarray(net.c, np.float32))
    assert np.array_equal(out, o_out)
    assert same_info(info, o_info) is None
    assert info["steps"].max() > 10_000


def test_config2_full_batch_plan_and_graph():
    """64 x 128 synthetic network, the full 65,536-simulation batch at t_end 10
    and 200 samples, on the library's plan for that batch (the kernel
    compiled for the network), launched through a captured CUDA graph
    (twice); 64 simulations spread over the batch are compared with the
    oracle, and a 512-simulation window run by the library's own kernel
    with the graph's rows."""
    net = inputs.synthetic(64, 128, 65536, seed=0, t_end=10.0, samples=200)
    model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    li, kw = _plan_cfg(model, net.n, 1, 1)
    assert li.specialized == 1, "the full batch runs the kernel compiled for the network"
    out, info = _device(net, model, 0, net.n, 1, kw, graph=True)
    idx = np.linspace(0, net.n - 1, 64).astype(np.int64)
    o_info = _compare(net, out, info, 0, idx, 1, f"config 2 (G={li.group}, min_blocks={li.min_blocks})")
    assert o_info["steps"].min() > 20_000   # full-length trajectories
    # the graph's results equal the library kernel's on a window
    out2, info2 = _device(net, model, 30000, 30512, 1, dict(kw, spec=-1))
    assert np.array_equal(out2, out[30000:30512])
    assert same_info(info2, info[30000:30512]) is None


@pytest.mark.parametrize("sched", [1, 2])
def test_config3_segments_with_perturbed_rates(sched):
    """The uneven batch's two segments (2^19 simulations each) with their
    log-normally perturbed rate constants: a 65,536-simulation window from the
    middle of each segment on the segment's full-batch plan, in both
    scheduling modes (the autotuner may pick either); 48 simulations spread
    over each window are compared with the oracle."""
    import bench
    segs = bench.workload(3)
    for si, (net, _) in enumerate(segs):
        model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        lo, hi = 200_000, 200_000 + 65536
        _, kw = _plan_cfg(model, net.n, 1 + si, 0, sched=sched)
        out, info = _device(net, model, lo, hi, 1 + si, kw)
        idx = np.linspace(lo, hi - 1, 48).astype(np.int64)
        _compare(net, out, info, lo, idx, 1 + si, f"config 3 segment {si} sched {sched}")


def test_config4_large_sparse_network_multiwarp_groups():
    """512 x 1024 sparse network at t_end 20 and 500 samples on the library's
    plan for the full 16,384-simulation batch (whole warps per simulation, the
    kernel compiled for the network): a 1,184-simulation window, 16 of its
    simulations compared with the oracle."""
    net = inputs.synthetic(512, 1024, 16384, seed=0, t_end=20.0, samples=500, c_range=(1e-5, 1e-1),
                           x0_range=(1, 100000))
    model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    li, kw = _plan_cfg(model, net.n, 1, 1, spec=1)  # the full batch's kernel, compiled for the network
    assert li.group >= 64 and li.specialized == 1
    lo, hi = 9000, 9000 + 1184
    out, info = _device(net, model, lo, hi, 1, kw)
    idx = np.linspace(lo, hi - 1, 16).astype(np.int64)
    o_info = _compare(net, out, info, lo, idx, 1, f"config 4 (G={li.group})")
    assert o_info["leaps"].min() > 10_000
