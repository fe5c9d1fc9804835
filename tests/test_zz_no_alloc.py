"""The allocation-free entry point, ctl_run_device_noalloc.

It serves callers that may not allocate device memory themselves (their
memory comes from a pool they manage, or their budget is fixed), so it keeps
the model tables and the work-queue ticket in a fixed 1 MiB array inside the
library.  Its results must equal ctl_run_device's bit for bit, on two calls in
a row with different models (the second call reuses the array the first one
left filled).  The file name sorts last so that a run which stops at the first
failure has already run every other test; it also passes on its own.
"""
import ctypes as C

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs


def _device_run(model, net, entry, seed):
    import torch
    X0 = torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).cuda()
    out = torch.full((net.n, model.ns, model.s_out), -1, dtype=torch.int32, device="cuda")
    info = torch.zeros((net.n, 40), dtype=torch.uint8, device="cuda")
    cfg = ctl.run_cfg(seed=seed)
    st = entry(model.handle, C.byref(cfg), net.n, C.c_void_p(X0.data_ptr()), C.c_void_p(c.data_ptr()),
               C.c_void_p(out.data_ptr()), C.c_void_p(info.data_ptr()),
               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == ctl.OK, ctl.lib().ctl_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy(), info.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_on_two_calls():
    L = ctl.lib()
    nets = [inputs.synthetic(16, 32, 96, seed=7, t_end=1.0, samples=20, x0_range=(10, 2000), perturb_sigma=0.5,
                             perturb_seed=7),
            inputs.schlogl(64, samples=25, t_end=1.0)]
    for call, net in enumerate(nets):
        model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        got, got_info = _device_run(model, net, L.ctl_run_device_noalloc, seed=40 + call)
        ref, ref_info = _device_run(model, net, L.ctl_run_device, seed=40 + call)
        assert np.array_equal(got, ref), f"call {call}: samples differ"
        assert np.array_equal(got_info, ref_info), f"call {call}: records differ"


@pytest.mark.gpu
def test_noalloc_leaves_device_memory_unchanged():
    """The promise itself: a call allocates no device memory.  After a
    warm-up call of the same launch shape (which loads the kernel), a model
    that the allocating entry has never seen runs through the no-alloc entry
    with every buffer allocated beforehand, and the device's free memory is
    the same before and after; its results then equal ctl_run_device's."""
    import torch
    L = ctl.lib()
    net = inputs.synthetic(8, 12, 80, seed=21, t_end=0.8, samples=15, x0_range=(5, 500))
    warm = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    _device_run(warm, net, L.ctl_run_device_noalloc, seed=5)
    fresh = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
    X0 = torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).cuda()
    c = torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).cuda()
    out = torch.full((net.n, fresh.ns, fresh.s_out), -1, dtype=torch.int32, device="cuda")
    info = torch.zeros((net.n, 40), dtype=torch.uint8, device="cuda")
    cfg = ctl.run_cfg(seed=6)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    st = L.ctl_run_device_noalloc(fresh.handle, C.byref(cfg), net.n, C.c_void_p(X0.data_ptr()),
                                  C.c_void_p(c.data_ptr()), C.c_void_p(out.data_ptr()),
                                  C.c_void_p(info.data_ptr()), C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert st == ctl.OK, L.ctl_last_error()
    assert free_after == free_before, f"device memory changed by {free_before - free_after} bytes"
    ref, ref_info = _device_run(fresh, net, L.ctl_run_device, seed=6)
    assert np.array_equal(out.cpu().numpy(), ref)
    assert np.array_equal(info.cpu().numpy(), ref_info)


def test_noalloc_rejects_models_beyond_its_array():
    # 60000 reactions of two reactants: the packed tables alone exceed 1 MiB
    S, R = 200, 60000
    rng = np.random.default_rng(0)
    left = np.zeros((R, S), np.int32)
    right = np.zeros((R, S), np.int32)
    left[np.arange(R), rng.integers(0, S, R)] = 1
    left[np.arange(R), rng.integers(0, S, R)] += 1
    right[np.arange(R), rng.integers(0, S, R)] = 1
    model = ctl.Model.create(left, right, None, [1.0])
    cfg = ctl.run_cfg()
    st = ctl.lib().ctl_run_device_noalloc(model.handle, C.byref(cfg), 1, None, None, None, None, None)
    assert st == ctl.ERR_SHAPE
    assert b"1 MiB" in ctl.lib().ctl_last_error()
