"""GPU parity of the shared-memory sweep compiled for one network.

For batches of at least 4,096 simulations (or with ctl_run_cfg.spec = 1)
the library compiles the shared-memory sweep at run time with NVRTC, the
network's geometry (species, reactions, tree levels, sample counts) as
compile-time constants.  It must reproduce the CPU oracle (oracle/, the
restatement of PreCalculations, EventualSSASteps and LightweightSSA,
2phase_n-tau-leaping.cu:1568-2454) bit for bit, exactly as the library's own
kernels do: every sample and every per-simulation record field, across
group sizes, both scheduling modes, the register budgets, the quirk
switches and the fitness-mode sums.
"""
import ctypes as C

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs
from tests.netutil import oracle_run, same_info, small_networks

pytestmark = pytest.mark.gpu

# networks of the shared-memory sweep (the register-resident sweep takes the
# tiny ones unless a group size is given, which every call here does)
NETS = [(n, net) for n, net in small_networks() if n != "schlogl"]


def _model(net):
    return ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)


@pytest.mark.parametrize("name,net", NETS, ids=[n for n, _ in NETS])
def test_compiled_sweep_bit_exact(name, net):
    out_o, info_o = oracle_run(net, seed=321)
    m = _model(net)
    for G, sched in ((1, 1), (4, 2), (8, 1), (32, 2)):
        if G > m.launch_info(net.n, group=G, spec=-1).group:  # G is capped at the tree's leaves
            continue
        li = m.launch_info(net.n, group=G, sched=sched, spec=1)
        assert li.specialized == 1, f"{name} G={G}: no compiled kernel"
        out, info = m.run(net.X0, net.c, seed=321, group=G, sched=sched, spec=1)
        assert np.array_equal(out, out_o), f"{name} G={G} sched={sched}: samples differ"
        f = same_info(info, info_o)
        assert f is None, f"{name} G={G} sched={sched}: record field {f} differs"


def test_compiled_sweep_register_budgets_and_quirks():
    name, net = NETS[-2]  # per-simulation rates, quirk paths reached
    m = _model(net)
    for mb in (2, 3, 4):
        out_o, info_o = oracle_run(net, seed=5)
        out, info = m.run(net.X0, net.c, seed=5, group=8, min_blocks=mb, spec=1)
        assert m.launch_info(net.n, group=8, min_blocks=mb, spec=1).specialized == 1
        assert np.array_equal(out, out_o) and same_info(info, info_o) is None, f"{name} min_blocks={mb}"
    for flags in (ctl.FORCE_SSA, ctl.ALL_QUIRKS_OFF, ctl.Q2_OFF | ctl.Q3_OFF):
        out_o, info_o = oracle_run(net, seed=9, flags=flags)
        out, info = m.run(net.X0, net.c, seed=9, flags=flags, group=4, spec=1)
        assert np.array_equal(out, out_o) and same_info(info, info_o) is None, f"{name} flags={flags:#x}"


def test_compiled_sweep_multiwarp_groups():
    """Groups of 64 and 128 lanes (named barriers per group) on a network
    with more reactions than a warp has lanes."""
    net = inputs.synthetic(48, 160, 24, seed=13, t_end=0.3, samples=12, x0_range=(20, 4000))
    out_o, info_o = oracle_run(net, seed=77)
    m = _model(net)
    for G in (64, 128):
        out, info = m.run(net.X0, net.c, seed=77, group=G, spec=1)
        assert m.launch_info(net.n, group=G, spec=1).specialized == 1
        assert np.array_equal(out, out_o) and same_info(info, info_o) is None, f"G={G}"


def test_library_choice_of_the_compiled_sweep():
    """spec = 0 compiles for batches of at least 4,096 simulations, -1 never;
    both kernels give the same bits on a window of such a batch."""
    net = inputs.synthetic(16, 32, 4096, seed=7, t_end=0.2, samples=10, x0_range=(10, 2000))
    m = _model(net)
    assert m.launch_info(4096, group=4).specialized == 1
    assert m.launch_info(4095, group=4).specialized == 0
    assert m.launch_info(4096, group=4, spec=-1).specialized == 0
    a, ia = m.run(net.X0, net.c, seed=3, group=4)
    b, ib = m.run(net.X0, net.c, seed=3, group=4, spec=-1)
    assert np.array_equal(a, b) and same_info(ia, ib) is None
    out_o, info_o = oracle_run(inputs.Network(net.left, net.right, net.feed, net.X0[:40], net.c[:40], net.tvec,
                                              net.cs), seed=3)
    assert np.array_equal(a[:40], out_o) and same_info(ia[:40], info_o) is None


def test_compiled_sweep_fitness_sums():
    """Fitness mode (per-set sample sums in the kernel) on the compiled
    kernel equals the sums of the library kernel's stored samples."""
    import torch
    net = inputs.synthetic(16, 32, 256, seed=7, t_end=0.5, samples=12, x0_range=(10, 2000))
    m = _model(net)
    n, ns, so, threads, p_rep = net.n, len(net.tvec), net.S, 32, 4
    dev = lambda a: torch.as_tensor(a, device="cuda")
    X0, c = dev(np.ascontiguousarray(net.X0, np.int32)), dev(np.ascontiguousarray(net.c, np.float32))
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.empty(n * ns * so, dtype=torch.int32, device="cuda")
    info_a = torch.empty(n * 40, dtype=torch.uint8, device="cuda")
    m.run_device(n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info_a.data_ptr(), stream,
                 ctl.run_cfg(seed=4, group=4, spec=-1))
    sums = torch.full(((n // p_rep) * ns * so,), -1, dtype=torch.int64, device="cuda")
    info_b = torch.empty(n * 40, dtype=torch.uint8, device="cuda")
    cfg = ctl.run_cfg(seed=4, group=4, spec=1)
    P = C.c_void_p
    assert ctl.lib().ctl_run_device_sums(m._h, C.byref(cfg), n, P(X0.data_ptr()), P(c.data_ptr()), threads, p_rep,
                                         P(sums.data_ptr()), P(info_b.data_ptr()), P(stream)) == ctl.OK
    torch.cuda.synchronize()
    samples = out.cpu().numpy().view(np.uint32).reshape(n, ns, so).astype(np.uint64)
    gid = np.arange(n)
    sets = (gid // (threads * p_rep)) * threads + gid % threads
    ref = np.zeros((n // p_rep, ns, so), np.uint64)
    np.add.at(ref, sets, samples)
    assert np.array_equal(sums.cpu().numpy().view(np.uint64).reshape(n // p_rep, ns, so), ref)
    assert np.array_equal(info_a.cpu().numpy(), info_b.cpu().numpy())
