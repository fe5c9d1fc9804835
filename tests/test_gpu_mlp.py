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
