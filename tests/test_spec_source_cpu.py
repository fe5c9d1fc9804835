"""The network-compiled shared-memory sweep, checked without a GPU.

For large batches the library compiles the sweep of ctl_sweep_dev.cuh at run
time with NVRTC, the network's geometry as compile-time constants
(ctl_run_cfg.spec).  ctl_spec_source returns the source it compiles; NVRTC
needs no GPU, so this test compiles that source for sm_100a here -- with
the same options and the same device headers the library embeds -- for
networks whose trees have one, two and four stored levels, group sizes from
1 to 256 lanes and the three register budgets.  A compilation error would
otherwise only show on a GPU, as a silent fall-back to the library's own
kernel.
"""
import ctypes as C
import os

import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs

CSRC = os.path.join(os.path.dirname(ctl.__file__), "csrc")
HEADERS = ("ctl_devmath.cuh", "ctl_tiny_body.cuh", "ctl_sweep_dev.cuh")


def _nvrtc():
    for name in ("libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"):
        try:
            return C.CDLL(name)
        except OSError:
            pass
    pytest.skip("NVRTC is not installed")


def _compile(nv, src):
    """(status, log) of an NVRTC compilation with the library's options."""
    texts = [open(os.path.join(CSRC, h)).read().encode() for h in HEADERS]
    prog = C.c_void_p()
    H = (C.c_char_p * 3)(*texts)
    N = (C.c_char_p * 3)(*[h.encode() for h in HEADERS])
    assert nv.nvrtcCreateProgram(C.byref(prog), src.encode(), b"ctl_spec.cu", 3, H, N) == 0
    opts = [b"--gpu-architecture=sm_100a", b"-fmad=false", b"--std=c++17"]
    rc = nv.nvrtcCompileProgram(prog, len(opts), (C.c_char_p * len(opts))(*opts))
    n = C.c_size_t()
    nv.nvrtcGetProgramLogSize(prog, C.byref(n))
    log = C.create_string_buffer(n.value + 1)
    nv.nvrtcGetProgramLog(prog, log)
    cub = C.c_size_t()
    if rc == 0:
        nv.nvrtcGetCUBINSize(prog, C.byref(cub))
    nv.nvrtcDestroyProgram(C.byref(prog))
    return rc, log.value.decode(errors="replace"), cub.value


def _model(S, R, seed):
    net = inputs.synthetic(S, R, 4, seed=seed, t_end=1.0, samples=5)
    return ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)


@pytest.mark.parametrize("S,R,G,minb", [(4, 6, 1, 2), (64, 128, 8, 3), (64, 128, 8, 2), (64, 128, 32, 4),
                                        (512, 1024, 128, 3), (512, 1024, 256, 2)],
                         ids=["8leaves-G1", "cfg2-G8-b3", "cfg2-G8-b2", "cfg2-G32-b4", "cfg4-G128", "cfg4-G256"])
def test_spec_source_compiles_for_sm100a(S, R, G, minb):
    nv = _nvrtc()
    m = _model(S, R, seed=S)
    src = m.spec_source(G, minb)
    # the geometry is in the source as constants, the tables are not
    assert f"S = {S}, R = {R}" in src and f"__launch_bounds__(256, {minb})" in src
    assert f"sweep_body<{min(G, m.P)}>" in src
    rc, log, cubin = _compile(nv, src)
    assert rc == 0, log[-3000:]
    assert cubin > 0


def test_spec_source_arguments():
    m = _model(16, 32, seed=3)
    n = C.c_size_t()
    L = ctl.lib()
    for G, mb in ((3, 3), (512, 3), (8, 1), (8, 5), (0, 3)):
        assert L.ctl_spec_source(m._h, G, mb, None, 0, C.byref(n)) == ctl.ERR_ARG
    assert L.ctl_spec_source(m._h, 8, 3, None, 0, C.byref(n)) == ctl.OK and n.value > 100
    small = C.create_string_buffer(16)
    assert L.ctl_spec_source(m._h, 8, 3, small, 16, C.byref(n)) == ctl.ERR_SHAPE
    # the same geometry gives the same source; a different one does not
    assert m.spec_source(8) == _model(16, 32, seed=4).spec_source(8)
    assert m.spec_source(8) != _model(16, 48, seed=3).spec_source(8)
    assert "sweep_body<32>" in m.spec_source(64)  # capped at the tree's 32 leaves
