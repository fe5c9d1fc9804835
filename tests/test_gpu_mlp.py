"""The surrogate's tcgen05 kernels on the GPU.

* GEMM epilogues against a plain PyTorch FP32 matmul of the same BF16 values
  (tolerance: |err| <= 2e-3 * max|C| + 1e-3 for FP32 outputs, one BF16 ulp
  (2^-8 relative) for BF16 outputs);
* full-network gradients against the CPU FP32 oracle (oracle/mlp_oracle.py)
  which rounds to BF16 at the same points (relative Frobenius error <= 2e-2);
* a short training run reduces the negative log-likelihood.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (128, 64, 128), (256, 256, 256), (384, 128, 1024),
                                   (128, 512, 64)])
def test_gemm_f32_matches_torch(M, N, K):
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    out = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    sg.gemm(A, B, epilogue=sg.EPI_F32, out_f32=out, err=err)
    torch.cuda.synchronize()
    ref = A.float() @ B.float().t()
    assert int(err.item()) == 0
    assert torch.isfinite(out).all()
    assert (out - ref).abs().max().item() <= 2e-3 * ref.abs().max().item() + 1e-3


def test_gemm_split_k_atomic():
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(256, 4096, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(64, 4096, device="cuda", generator=g).to(torch.bfloat16)
    out = torch.zeros(256, 64, device="cuda")
    sg.gemm(A, B, epilogue=sg.EPI_ATOMIC_F32, out_f32=out, splits=16)
    torch.cuda.synchronize()
    ref = A.float() @ B.float().t()
    assert (out - ref).abs().max().item() <= 2e-3 * ref.abs().max().item() + 1e-3


def test_gemm_bias_silu_and_grad_epilogues():
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(3)
    M, N, K = 256, 128, 192
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16) * 0.3
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16) * 0.3
    bias = torch.randn(N, device="cuda", generator=g)
    z = torch.empty(M, N, device="cuda")
    h = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    hT = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
    sg.gemm(A, B, epilogue=sg.EPI_BIAS_SILU, out_f32=z, out_bf=h, out_bfT=hT, bias=bias)
    zr = A.float() @ B.float().t() + bias
    hr = torch.nn.functional.silu(zr)
    torch.cuda.synchronize()
    assert (z - zr).abs().max().item() <= 2e-3 * zr.abs().max().item() + 1e-3
    assert ((h.float() - hr).abs() <= hr.abs() * 2 ** -7 + 1e-2).all()
    assert torch.equal(hT, h.t())
    zin = torch.randn(M, N, device="cuda", generator=g)
    d = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    dT = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
    sg.gemm(A, B, epilogue=sg.EPI_SILU_GRAD, z_in=zin, out_bf=d, out_bfT=dT)
    s = torch.sigmoid(zin)
    dr = (A.float() @ B.float().t()) * s * (1 + zin * (1 - s))
    torch.cuda.synchronize()
    assert ((d.float() - dr).abs() <= dr.abs() * 2 ** -7 + 2e-2).all()
    assert torch.equal(dT, d.t())


def test_mlp_gradients_match_cpu_oracle():
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    from oracle import mlp_oracle as mo
    S, Bn = 32, 512
    net = sg.MLP(S, seed=1)
    rng = np.random.default_rng(0)
    X = np.zeros((Bn, sg.IN_PAD), np.float32)
    X[:, :9] = rng.uniform(-1, 1, (Bn, 9))
    tgt = rng.normal(0, 1, (Bn, S)).astype(np.float32)
    Xg = torch.from_numpy(X).cuda().to(torch.bfloat16)
    y = net.forward(Xg)
    loss, dW, db = net.backward(y, torch.from_numpy(tgt).cuda())
    torch.cuda.synchronize()
    net.check_error_flag()
    W = [w.cpu().numpy() for w in net.W]
    b = [x.cpu().numpy() for x in net.b]
    l_o, dW_o, db_o, y_o = mo.backward(X, W, b, tgt)
    assert np.allclose(y.cpu().numpy(), y_o, rtol=2e-2, atol=2e-3)
    assert net.out_w == 64 and np.all(W[-1][2 * S:] == 0)
    assert abs(loss.item() - l_o) / abs(l_o) < 1e-3
    for l in range(len(W)):
        g, o = dW[l].cpu().numpy(), dW_o[l]
        assert np.linalg.norm(g - o) <= 2e-2 * np.linalg.norm(o) + 1e-7, f"dW[{l}]"
        g, o = db[l].cpu().numpy(), db_o[l]
        assert np.linalg.norm(g - o) <= 2e-2 * np.linalg.norm(o) + 1e-7, f"db[{l}]"


def test_mlp_training_reduces_nll():
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    S, Bn = 16, 2048
    net = sg.MLP(S, seed=2)
    g = torch.Generator(device="cuda").manual_seed(5)
    losses = []
    for it in range(300):
        X = torch.zeros(Bn, sg.IN_PAD, device="cuda")
        X[:, :9] = torch.rand(Bn, 9, device="cuda", generator=g) * 2 - 1
        k = torch.arange(S, device="cuda", dtype=torch.float32)
        mean = torch.sin(X[:, :1] * (1 + k / 4) + X[:, 1:2]) + 0.5 * X[:, 2:3]
        tgt = mean + 0.1 * torch.randn(Bn, S, device="cuda", generator=g)
        y = net.forward(X.to(torch.bfloat16))
        loss, dW, db = net.backward(y, tgt)
        net.adam(dW, db, lr=2e-3)
        losses.append(loss.item() / (Bn * S))
    net.check_error_flag()
    assert np.mean(losses[-20:]) < np.mean(losses[:20]) - 1.0, (losses[:3], losses[-3:])


def _screen_setup(S, n_cand, ns, seed):
    """A surrogate with random biases, a candidate set, instants and a
    target (one zero entry: the absolute-difference branch)."""
    import math
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    net = sg.MLP(S, seed=seed)
    g = torch.Generator(device="cuda").manual_seed(seed)
    for l in range(len(net.b)):
        net.b[l].copy_(0.2 * torch.randn(net.b[l].shape, device="cuda", generator=g))
    rng = np.random.default_rng(seed)
    lo, hi = np.full(8, math.log(1e-3)), np.zeros(8)
    sc = sg.Scaling(lo, hi, 5.0, rng.uniform(50, 500, S).astype(np.float32),
                    rng.uniform(5, 50, S).astype(np.float32))
    theta = rng.uniform(lo, hi, size=(n_cand, 8)).astype(np.float32)
    tvec = (5.0 * np.arange(1, ns + 1) / ns).astype(np.float32)
    target = rng.integers(1, 800, size=(ns, S)).astype(np.float32)
    target[0, 0] = 0.0
    return net, sc, theta, tvec, target


def _fitness_of_mean(mean, target):
    d = np.abs(target[None].astype(np.float64) - mean)
    d = np.where(target[None] != 0, d / np.maximum(target[None], 1), d)
    return d.sum(axis=(1, 2)) / (target.shape[0] * target.shape[1])


@pytest.mark.parametrize("S,n_cand,ns", [(5, 37, 7), (16, 1, 1), (32, 130, 1), (32, 9, 50)])
def test_screen_matches_cpu_oracle(S, n_cand, ns):
    """Fused screening (input build, five layers, fitness) against the CPU
    oracle's forward pass with the same BF16 rounding; tolerance 2e-3
    relative on each candidate's fitness (BF16 ties may round differently
    under FP32 vs FP64 accumulation)."""
    torch = _torch()
    import oracle.mlp_oracle as mo
    from cutauleaping_b200 import surrogate as sg
    net, sc, theta, tvec, target = _screen_setup(S, n_cand, ns, seed=S + n_cand + ns)
    fit = sg.screen(net, torch.as_tensor(theta, device="cuda"), tvec, target, sc)
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    # oracle input rows: the same FP32 operations, then BF16
    f32 = np.float32
    th = np.repeat(theta, ns, axis=0)
    tt = np.tile(tvec, n_cand)
    X = np.zeros((n_cand * ns, 64), dtype=f32)
    X[:, :8] = (f32(2.0) * (th - sc.log_lo.astype(f32))) / (sc.log_hi.astype(f32) - sc.log_lo.astype(f32)) - f32(1.0)
    X[:, 8] = (f32(2.0) * tt) / f32(sc.t_end) - f32(1.0)
    W = [w.cpu().numpy() for w in net.W]
    b = [x.cpu().numpy() for x in net.b]
    y, _, _ = mo.forward(X, W, b)
    mean = (y[:, :S].astype(np.float64) * sc.y_std + sc.y_mean).reshape(n_cand, ns, S)
    ref = _fitness_of_mean(mean, target)
    got = fit.cpu().numpy()
    assert np.allclose(got, ref, rtol=2e-3, atol=1e-6), np.abs(got / ref - 1).max()


def test_screen_matches_layered_path():
    """Many tiles per CTA: the fused kernel against the layer-by-layer tcgen05
    GEMM path on the same network (same MMA sequence per layer, so the hidden
    activations agree; the last step differs only by FP32 vs FP64): 1e-5."""
    torch = _torch()
    from cutauleaping_b200 import surrogate as sg
    S, n_cand, ns = 32, 3001, 50
    net, sc, theta, tvec, target = _screen_setup(S, n_cand, ns, seed=11)
    th = torch.as_tensor(theta, device="cuda")
    fit = sg.screen(net, th, tvec, target, sc).cpu().numpy()
    rows = n_cand * ns
    pad = (-rows) % 128
    X = sg.make_inputs(th.repeat_interleave(ns, 0), torch.as_tensor(tvec, device="cuda").repeat(n_cand), sc, torch)
    X = torch.cat([X, torch.zeros(pad, X.shape[1], dtype=X.dtype, device="cuda")])
    y = net.forward(X, keep=False)[:rows, :S].double().cpu().numpy()
    mean = (y * sc.y_std.astype(np.float64) + sc.y_mean.astype(np.float64)).reshape(n_cand, ns, S)
    ref = _fitness_of_mean(mean, target)
    assert int(net.err.item()) == 0
    assert np.allclose(fit, ref, rtol=1e-5, atol=1e-9), np.abs(fit / ref - 1).max()


def test_bounded_wait_gives_up_and_reports():
    """The kernels' bounded mbarrier wait, on a barrier that nothing arrives
    on (nothing in flight): it gives up after its poll limit, raises the
    error word, the kernel returns (the context stays usable), and the
    surrogate's host check turns the raised word into an error."""
    import ctypes as C
    import torch
    import cutauleaping_b200 as ctl
    L = ctl.lib()
    L.ctl_mlp_wait_check.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = L.ctl_mlp_wait_check(C.c_void_p(err.data_ptr()), 4096, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == ctl.OK
    torch.cuda.synchronize()
    assert int(err.item()) == 3
    assert L.ctl_mlp_wait_check(C.c_void_p(err.data_ptr()), 0, None) == ctl.ERR_ARG
    # the context is still usable and the host side reports a raised word
    from cutauleaping_b200 import surrogate as sg
    net = sg.MLP(4, seed=0)
    net.err.fill_(1)
    with pytest.raises(RuntimeError):
        net.check_error_flag()
    net.err.zero_()
    net.check_error_flag()
