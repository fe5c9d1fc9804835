"""GPU parity: the CUDA sweep reproduces the CPU oracle bit for bit.

Every test calls the product through its C ABI (libctl.so via ctypes) and
compares against oracle/ (the C restatement of PreCalculations,
EventualSSASteps and LightweightSSA, 2phase_n-tau-leaping.cu:1568-2454) on the
same seeded inputs.  Samples and per-simulation counters are integers and are
compared exactly; t_final is an FP64 value produced by the same sequence of
IEEE operations and is compared exactly as well.
"""
import numpy as np
import pytest

import cutauleaping_b200 as ctl
from tests.netutil import oracle_run, same_info, small_networks

pytestmark = pytest.mark.gpu

NETS = small_networks()


def gpu_run(net, **kw):
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    return m.run(net.X0, net.c, **kw)


@pytest.mark.parametrize("name,net", NETS, ids=[n for n, _ in NETS])
def test_bit_exact_vs_oracle(name, net):
    out_o, info_o = oracle_run(net, seed=123)
    out_g, info_g = gpu_run(net, seed=123)
    assert np.array_equal(out_g, out_o), f"{name}: samples differ"
    assert same_info(info_g, info_o) is None, f"{name}: info field {same_info(info_g, info_o)} differs"
    assert (info_g["status"] == ctl.SIM_OK).all()


@pytest.mark.parametrize("flags", [ctl.FORCE_SSA, ctl.Q1_OFF, ctl.Q2_OFF, ctl.Q3_OFF, ctl.Q4_OFF,
                                   ctl.Q5_OFF, ctl.Q6_OFF, ctl.Q9_OFF, ctl.Q10_OFF,
                                   ctl.ALL_QUIRKS_OFF, ctl.ALL_QUIRKS_OFF | ctl.FORCE_SSA])
def test_quirk_switches_bit_exact(flags):
    for name, net in NETS[:4]:
        out_o, info_o = oracle_run(net, seed=7, flags=flags)
        out_g, info_g = gpu_run(net, seed=7, flags=flags)
        assert np.array_equal(out_g, out_o), f"{name} flags={flags:#x}"
        assert same_info(info_g, info_o) is None, f"{name} flags={flags:#x}"


@pytest.mark.parametrize("name,net", NETS, ids=[n for n, _ in NETS])
def test_launch_shape_invariance(name, net):
    ref, ref_info = gpu_run(net, seed=99, group=1, threads=256)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    for G in (1, 2, 4, 8, 16, 32):
        for threads in (32, 96, 256):
            if threads % G:
                continue
            out, info = m.run(net.X0, net.c, seed=99, group=G, threads=threads)
            assert np.array_equal(out, ref), f"{name} G={G} threads={threads}"
            assert same_info(info, ref_info) is None, f"{name} G={G} threads={threads}"


@pytest.mark.parametrize("name,net", NETS, ids=[n for n, _ in NETS])
def test_register_budget_invariance(name, net):
    """The register-budget variants (min_blocks 2, 3 and 4; the tighter ones
    spill to local memory) run the same arithmetic: identical to the oracle."""
    out_o, info_o = oracle_run(net, seed=31)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    for mb in (2, 3, 4):
        for G in (1, 8):
            out, info = m.run(net.X0, net.c, seed=31, group=G, min_blocks=mb)
            assert np.array_equal(out, out_o), f"{name} G={G} min_blocks={mb}"
            assert same_info(info, info_o) is None, f"{name} G={G} min_blocks={mb}"
            assert m.launch_info(net.n, group=G, min_blocks=mb).min_blocks == mb


@pytest.mark.parametrize("name,net", NETS, ids=[n for n, _ in NETS])
def test_warp_local_scheduling_invariance(name, net):
    """Warp-local scheduling (no block rounds) changes only which warp runs a
    simulation when: identical to the oracle for every group size."""
    out_o, info_o = oracle_run(net, seed=47)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    for G in (1, 4, 32):
        for threads in (32, 256):
            out, info = m.run(net.X0, net.c, seed=47, group=G, threads=threads, sched=2, ssa_budget=3)
            assert np.array_equal(out, out_o), f"{name} G={G} threads={threads}"
            assert same_info(info, info_o) is None, f"{name} G={G} threads={threads}"
    assert m.launch_info(net.n, sched=2).sched == 2


TINY = [(n, net) for n, net in NETS if n in ("schlogl", "syn4x6", "syn8x12p", "feed3")]


@pytest.mark.parametrize("name,net", TINY, ids=[n for n, _ in TINY])
def test_register_resident_sweep_bit_exact(name, net):
    """The register-resident sweep for tiny networks (one thread per
    simulation, everything in registers) reproduces the oracle bit for bit
    for any number of simulations per warp, block size and SSA budget, both
    in the kernel compiled at run time for the network (NVRTC) and in the
    library's own; the compiled one is the library's choice."""
    out_o, info_o = oracle_run(net, seed=61)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    li = m.launch_info(net.n)
    assert li.warp_sims > 0 and li.specialized == 1
    assert m.launch_info(net.n, spec=-1).specialized == 0
    assert m.launch_info(net.n, group=4).warp_sims == 0
    # sched 2: warp lockstep; sched 1: block rounds regrouping the simulations by phase
    shapes = [(2, ws, th) for ws in (1, 3, 8, 32) for th in (32, 256)] + \
             [(1, ws, th) for ws, th in ((1, 64), (3, 64), (16, 64), (5, 128), (32, 256))]
    for spec in (0, -1):   # the kernel compiled for this network, the library's own
        for sched, ws, threads in shapes:
            for sb, db in ((1, 1), (16, 2)):
                out, info = m.run(net.X0, net.c, seed=61, warp_sims=ws, threads=threads, ssa_budget=sb,
                                  dec_budget=db, sched=sched, spec=spec)
                what = f"{name} spec={spec} sched={sched} warp_sims={ws} threads={threads} ssa_budget={sb}"
                assert np.array_equal(out, out_o), what
                assert same_info(info, info_o) is None, what
                li = m.launch_info(net.n, warp_sims=ws, threads=threads, sched=sched)
                assert li.warp_sims == ws and li.sched == sched


@pytest.mark.parametrize("flags", [ctl.FORCE_SSA, ctl.Q1_OFF, ctl.Q2_OFF, ctl.Q3_OFF, ctl.Q4_OFF,
                                   ctl.Q5_OFF, ctl.Q6_OFF, ctl.Q9_OFF, ctl.Q10_OFF,
                                   ctl.ALL_QUIRKS_OFF, ctl.ALL_QUIRKS_OFF | ctl.FORCE_SSA])
def test_register_resident_quirk_switches(flags):
    for name, net in TINY:
        out_o, info_o = oracle_run(net, seed=8, flags=flags)
        m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        for spec in (0, -1):
            for sched in (1, 2):
                out, info = m.run(net.X0, net.c, seed=8, flags=flags, warp_sims=4, spec=spec, sched=sched)
                assert np.array_equal(out, out_o), f"{name} flags={flags:#x} spec={spec} sched={sched}"
                assert same_info(info, info_o) is None, f"{name} flags={flags:#x} spec={spec} sched={sched}"


def test_register_resident_step_limit_and_sim_base():
    name, net = TINY[0]
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    out_o, _ = oracle_run(net, seed=1, max_steps=50)
    for sched in (1, 2):
        out, info = m.run(net.X0, net.c, seed=1, max_steps=50, check=False, warp_sims=2, sched=sched)
        assert (info["status"] == ctl.SIM_STEP_LIMIT).all() and (info["steps"] == 50).all()
        assert np.array_equal(out, out_o)
        full, _ = m.run(net.X0, net.c, seed=5, warp_sims=8, sched=sched)
        part, _ = m.run(net.X0[10:30], net.c[10:30], seed=5, sim_base=10, warp_sims=8, sched=sched)
        assert np.array_equal(part, full[10:30])


def test_register_resident_lone_simulations_and_register_budget():
    """Batches smaller than a block: a block whose work queue is closed
    finishes a lone simulation in warp lockstep.  The kernel compiled for the
    network at register budgets 1 (the default) and 2, under both scheduling
    modes: identical to the oracle.  Budget 1 is refused by the shared-memory
    sweep."""
    name, net = TINY[0]
    out_o, info_o = oracle_run(net, seed=23)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    assert m.launch_info(net.n).min_blocks == 1
    for n in (1, 2, 5, 33):
        for sched in (1, 2):
            for mb in (1, 2):
                out, info = m.run(net.X0[:n], net.c[:n], seed=23, sched=sched, min_blocks=mb)
                what = f"{name} n={n} sched={sched} min_blocks={mb}"
                assert np.array_equal(out, out_o[:n]), what
                assert same_info(info, info_o[:n]) is None, what
                assert m.launch_info(n, sched=sched, min_blocks=mb).min_blocks == mb
    with pytest.raises(ctl.CtlError) as e:
        m.run(net.X0, net.c, seed=23, group=4, min_blocks=1)
    assert e.value.status == ctl.ERR_ARG


def test_register_resident_refuses_larger_networks():
    name, net = [x for x in NETS if x[0] == "syn16x32"][0]
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    assert m.launch_info(net.n).warp_sims == 0
    with pytest.raises(ctl.CtlError):
        m.launch_info(net.n, warp_sims=4)


def test_uneven_batch_as_one_graph_matches_separate_runs():
    """Two batches of different networks (Schlogl on the register-resident
    sweep, a perturbed 16 x 32 network on the shared-memory sweep) as the
    parallel branches of one graph: each branch's results equal its own
    separate run and the oracle, on two launches of the graph."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    nets = [NETS[0][1], [x for x in NETS if x[0] == "syn16x32"][0][1]]
    parts, refs = [], []
    for i, net in enumerate(nets):
        m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        X0 = torch.as_tensor(np.ascontiguousarray(net.X0, np.int32), device="cuda")
        c = torch.as_tensor(np.ascontiguousarray(net.c, np.float32), device="cuda")
        out = torch.full((net.n, m.ns, m.s_out), -1, dtype=torch.int32, device="cuda")
        info = torch.zeros((net.n, 40), dtype=torch.uint8, device="cuda")
        cfg = ctl.run_cfg(seed=13 + i, uniform_rates=int(bool((net.c == net.c[0]).all())))
        parts.append((m, net.n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(), cfg))
        refs.append((m, X0, c, out, info))
        ref_o, ref_i = m.run(net.X0, net.c, seed=13 + i)
        orc_o, orc_i = oracle_run(net, seed=13 + i)
        assert np.array_equal(ref_o, orc_o)
        refs[-1] += (ref_o, ref_i)
    g = ctl.graph_multi(parts, stream)
    for _ in range(2):
        for r in refs:
            r[3].fill_(-1)
            r[4].zero_()
        g.launch(stream)
        torch.cuda.synchronize()
        for r in refs:
            assert np.array_equal(r[3].cpu().numpy().view(np.uint32), r[5])
            assert np.array_equal(r[4].cpu().numpy(), r[6].view(np.uint8).reshape(-1, 40))
    with pytest.raises(ctl.CtlError):   # one model twice would share its queue ticket
        ctl.graph_multi([parts[0], parts[0]], stream)
    del g


def test_sim_base_selects_rows_of_a_larger_run():
    """The reference's `offset` shards rows; with sim_base the shard reproduces
    the same simulations a single large run produces."""
    name, net = NETS[1]
    full, _ = gpu_run(net, seed=5)
    part, _ = gpu_run(net.subset(slice(10, 30)), seed=5, sim_base=10)
    assert np.array_equal(part, full[10:30])


def test_step_limit_status_without_hang():
    name, net = NETS[0]
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    out, info = m.run(net.X0, net.c, seed=1, max_steps=50, check=False)
    assert (info["status"] == ctl.SIM_STEP_LIMIT).all()
    assert (info["steps"] == 50).all()
    out_o, info_o = oracle_run(net, seed=1, max_steps=50)
    assert np.array_equal(out, out_o)
    with pytest.raises(ctl.CtlError):
        m.run(net.X0, net.c, seed=1, max_steps=50)


def test_multiwarp_groups_bit_exact():
    """Groups of 64, 128 and 256 lanes (whole warps per simulation, named
    barriers and shared-memory reductions) on a 64 x 200 network (256 tree
    leaves), under both scheduling modes: identical to the oracle."""
    from cutauleaping_b200 import inputs
    net = inputs.synthetic(64, 200, 24, seed=13, t_end=0.3, samples=10, x0_range=(10, 5000),
                           perturb_sigma=0.5, perturb_seed=13)
    out_o, info_o = oracle_run(net, seed=71)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    for G, threads in ((64, 128), (64, 256), (128, 256), (256, 256)):
        for sched in (1, 2):
            out, info = m.run(net.X0, net.c, seed=71, group=G, threads=threads, sched=sched)
            assert np.array_equal(out, out_o), f"G={G} threads={threads} sched={sched}"
            assert same_info(info, info_o) is None, f"G={G} threads={threads} sched={sched}"
            assert m.launch_info(net.n, group=G, threads=threads).group == G


def test_host_run_with_overlapped_copies_matches_device_run():
    """ctl_run copies finished chunks back while the sweep runs (batches with
    64 MB of samples or more): its rows and records equal a device-resident
    run's, and sampled rows equal the oracle's."""
    import torch
    from cutauleaping_b200 import inputs
    net = inputs.synthetic(64, 128, 2304, seed=0, t_end=0.4, samples=200)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    assert 2304 * 200 * 64 * 4 >= 64 << 20
    out_h, info_h = m.run(net.X0, net.c, seed=3)
    X0 = torch.as_tensor(np.ascontiguousarray(net.X0, np.int32), device="cuda")
    c = torch.as_tensor(np.ascontiguousarray(net.c, np.float32), device="cuda")
    out = torch.empty((net.n, 200, 64), dtype=torch.int32, device="cuda")
    info = torch.empty((net.n, 40), dtype=torch.uint8, device="cuda")
    m.run_device(net.n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(),
                 torch.cuda.current_stream().cuda_stream,
                 ctl.run_cfg(seed=3, uniform_rates=int(bool((net.c == net.c[0]).all()))))
    torch.cuda.synchronize()
    assert np.array_equal(out_h, out.cpu().numpy().view(np.uint32))
    assert np.array_equal(info_h.view(np.uint8).reshape(net.n, 40), info.cpu().numpy())
    sub = net.subset(slice(2300, 2304))
    out_o, info_o = oracle_run(sub, seed=3, sim_base=2300)
    assert np.array_equal(out_h[2300:2304], out_o)


def test_host_run_into_pinned_buffers_writes_rows_from_the_kernel():
    """With pinned (device-addressable) host buffers, ctl_run's kernel copies
    each finished row into the caller's buffer itself: the rows and records
    equal a device-resident run's, on the shared-memory sweep (rows of a
    multiple of four words, 16-byte stores) and on the register-resident one
    (Schlogl, 25 instants x 3 species: word stores)."""
    import ctypes as C
    import torch
    from cutauleaping_b200 import inputs
    L = ctl.lib()
    for net, kw in ((inputs.synthetic(16, 32, 200, seed=7, t_end=0.5, samples=12, perturb_sigma=0.5, perturb_seed=7),
                     {"group": 4}),
                    (inputs.schlogl(300, samples=25, t_end=1.0), {})):
        m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        cfg = ctl.run_cfg(seed=21, **kw)
        hX = torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).pin_memory()
        hc = torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).pin_memory()
        hout = torch.full((net.n, m.ns, m.s_out), -1, dtype=torch.int32).pin_memory()
        hinfo = torch.zeros((net.n, 40), dtype=torch.uint8).pin_memory()
        st = L.ctl_run(m.handle, C.byref(cfg), net.n, C.c_void_p(hX.data_ptr()), C.c_void_p(hc.data_ptr()),
                       C.c_void_p(hout.data_ptr()), C.c_void_p(hinfo.data_ptr()))
        assert st == ctl.OK, L.ctl_last_error()
        ref, ref_info = m.run(net.X0, net.c, cfg)          # pageable buffers: copies after the sweep
        assert np.array_equal(hout.numpy().view(np.uint32), ref)
        assert np.array_equal(hinfo.numpy(), ref_info.view(np.uint8).reshape(-1, 40))


def test_autotune_caches_a_shape_and_keeps_results():
    """ctl_autotune times the library's plan and its candidates, caches the
    winner for this batch size, and later calls with group == threads == 0
    run that shape with the same results as the untuned plan."""
    import torch
    from cutauleaping_b200 import inputs
    net = inputs.schlogl(3000, samples=20, t_end=2.0)
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    cfg = ctl.run_cfg(seed=17)
    before = m.launch_info(net.n, cfg)
    ref, ref_info = m.run(net.X0, net.c, cfg)
    X0 = torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).cuda()
    best = m.autotune(net.n, X0.data_ptr(), c.data_ptr(), sample=64, cfg=cfg)
    after = m.launch_info(net.n, cfg)
    for f in ("group", "threads", "min_blocks", "sched", "ssa_budget", "dec_budget"):
        assert getattr(after, f) == getattr(best, f), f
    assert best.group in (1, 2, 4) and best.min_blocks in (1, 2, 3, 4) and best.sched in (1, 2)
    out, info = m.run(net.X0, net.c, cfg)
    assert np.array_equal(out, ref) and same_info(info, ref_info) is None
    assert before.group >= 1
