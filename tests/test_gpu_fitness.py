"""Fitness mode without per-simulation samples on the GPU.

The fused path (ctl_run_device_sums + ctl_fitness_sums_device, and the
host-buffer ctl_fitness_run the CLI uses) adds every recorded sample into
64-bit per-set sums instead of storing it.  calculateFitness
(2phase_n-tau-leaping.cu:3324-3408) from those sums must equal, bit for bit,
calculateFitness from the stored samples (ctl_run_device +
ctl_fitness_device), including the A0 = 0 copy-forward of the last recorded
sample (tau.cu:1665-1697), both scheduling modes of the shared-memory sweep
and the register-resident sweep for tiny networks.
"""
import ctypes as C

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs

pytestmark = pytest.mark.gpu


def _decay_net(n):
    """X -> 0 and 2X -> 0 from small counts: most simulations go extinct
    before the end (A0 = 0, copy-forward of the last sample)."""
    left = np.array([[1], [2]], np.int32)
    right = np.array([[0], [0]], np.int32)
    X0 = np.tile(np.array([12], np.int32), (n, 1))
    c = np.tile(np.array([1.5, 0.05]), (n, 1))
    return inputs.Network(left, right, np.zeros(1, np.int32), X0, c, np.linspace(0.2, 6.0, 30),
                          np.array([0], np.int32))


def _both_paths(net, threads, p_rep, E, REP, seed, **cfgkw):
    import torch
    L = ctl.lib()
    n = net.n
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    ns, so = len(net.tvec), (net.S if net.cs is None else len(net.cs))
    blocks = n // threads
    rng = np.random.default_rng(seed)
    target = rng.integers(0, 300, size=(ns, E, REP, so)).astype(np.uint32)
    swarm = (np.arange(n) % E).astype(np.uint8)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    X0 = dev(np.ascontiguousarray(net.X0, np.int32))
    c = dev(np.ascontiguousarray(net.c, np.float32))
    tg, sw = dev(target.view(np.int32).reshape(-1)), dev(swarm)
    cfg = ctl.run_cfg(seed=seed, **cfgkw)
    stream = torch.cuda.current_stream().cuda_stream
    P = C.c_void_p
    # stored samples -> fitness
    out = torch.empty(n * ns * so, dtype=torch.int32, device="cuda")
    info_a = torch.empty(n * 40, dtype=torch.uint8, device="cuda")
    m.run_device(n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info_a.data_ptr(), stream, cfg)
    fa = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert L.ctl_fitness_device(P(out.data_ptr()), ns, so, P(tg.data_ptr()), P(sw.data_ptr()), E, REP, threads,
                                blocks, p_rep, P(fa.data_ptr()), P(stream)) == ctl.OK
    # per-set sums -> fitness
    sums = torch.full(((n // p_rep) * ns * so,), -1, dtype=torch.int64, device="cuda")
    info_b = torch.empty(n * 40, dtype=torch.uint8, device="cuda")
    assert L.ctl_run_device_sums(m._h, C.byref(cfg), n, P(X0.data_ptr()), P(c.data_ptr()), threads, p_rep,
                                 P(sums.data_ptr()), P(info_b.data_ptr()), P(stream)) == ctl.OK
    fb = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert L.ctl_fitness_sums_device(P(sums.data_ptr()), ns, so, P(tg.data_ptr()), P(sw.data_ptr()), E, REP,
                                     threads, blocks, p_rep, P(fb.data_ptr()), P(stream)) == ctl.OK
    torch.cuda.synchronize()
    samples = out.cpu().numpy().view(np.uint32).reshape(n, ns, so).astype(np.uint64)
    # the sums are exactly the per-set sums of the stored samples
    gid = np.arange(n)
    sets = (gid // (threads * p_rep)) * threads + gid % threads
    ref_sums = np.zeros((n // p_rep, ns, so), np.uint64)
    np.add.at(ref_sums, sets, samples)
    return (fa.cpu().numpy(), fb.cpu().numpy(), info_a.cpu().numpy(), info_b.cpu().numpy(),
            sums.cpu().numpy().view(np.uint64).reshape(n // p_rep, ns, so), ref_sums, samples)


@pytest.mark.parametrize("which", ["schlogl", "decay", "syn"])
@pytest.mark.parametrize("sched,warp_sims", [(1, -1), (2, -1), (2, 4), (1, 8)],
                         ids=["block-rounds", "warp-local", "register-resident", "register-resident-rounds"])
def test_sums_fitness_equals_sample_fitness(which, sched, warp_sims):
    if which == "schlogl":
        net, threads, p_rep = inputs.schlogl(96, samples=20, t_end=1.0), 8, 3
    elif which == "decay":
        net, threads, p_rep = _decay_net(64), 4, 4
    else:
        net = inputs.synthetic(16, 32, 72, seed=7, t_end=1.0, samples=15, x0_range=(10, 2000),
                               perturb_sigma=0.5, perturb_seed=7)
        threads, p_rep = 6, 2
    if warp_sims > 0 and which == "syn":
        pytest.skip("16 x 32 is beyond the register-resident sweep's limits")
    fa, fb, ia, ib, sums, ref, samples = _both_paths(net, threads, p_rep, E=2, REP=2, seed=17, sched=sched,
                                                     warp_sims=warp_sims)
    assert np.array_equal(sums, ref)
    assert np.array_equal(ia, ib)
    nsets = net.n // p_rep
    assert np.array_equal(fa[:nsets], fb[:nsets])
    if which == "decay":
        # extinction before the end: the last recorded (nonzero) sample was
        # copied forward to the remaining instants
        tail = samples[:, -5:, 0]
        assert ((tail == tail[:, :1]).all(axis=1) & (tail[:, 0] > 0)).any()


def test_fitness_run_rejects_bad_grouping():
    net = inputs.schlogl(12, samples=5, t_end=0.1)
    L = ctl.lib()
    m = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    cfg = ctl.run_cfg(seed=1)
    # n = 12 is not threads (5) * blocks
    st = L.ctl_run_device_sums(m._h, C.byref(cfg), 12, C.c_void_p(8), C.c_void_p(8), 5, 1, C.c_void_p(8),
                               C.c_void_p(8), None)
    assert st == ctl.ERR_ARG
