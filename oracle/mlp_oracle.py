"""CPU FP32 oracle of the surrogate MLP -- TEST INFRASTRUCTURE ONLY.

Forward and backward of the 9 -> 256 x 4 -> 2S SiLU network with the Gaussian
negative log-likelihood, in numpy float32 (float64 accumulation), rounding to
BF16 exactly where the GPU path stores BF16 (inputs, weights, hidden
activations, output gradient dY, hidden gradients dZ).  The GPU gradients
(tcgen05 GEMMs, split-K atomics) must agree within the tolerance the tests
state.
"""
import numpy as np


def bf16(x):
    """Round float32 to bfloat16 (round to nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(X, W, b):
    """X [B][64] (BF16 values), W[l] [out][in], b[l] [out] -> (y, zs, hs)."""
    h = bf16(X)
    hs, zs = [h], []
    for l in range(len(W) - 1):
        z = (h.astype(np.float64) @ bf16(W[l]).T.astype(np.float64) + b[l]).astype(np.float32)
        zs.append(z)
        h = bf16(silu(z))
        hs.append(h)
    y = (h.astype(np.float64) @ bf16(W[-1]).T.astype(np.float64) + b[-1]).astype(np.float32)
    return y, zs, hs


def nll_grad(y, tgt):
    """y = [mu | log var | zero padding]; the padding columns get zero gradient."""
    Bn, S = tgt.shape
    mu, lv = y[:, :S], np.clip(y[:, S:2 * S], -12.0, 12.0)
    iv = np.exp(-lv)
    d = tgt - mu
    loss = float((0.5 * (lv + d * d * iv)).sum())
    sc = 1.0 / (Bn * S)
    dy = np.zeros_like(y)
    dy[:, :S] = -d * iv * sc
    dy[:, S:2 * S] = 0.5 * (1.0 - d * d * iv) * sc
    return loss, bf16(dy)


def backward(X, W, b, tgt):
    """Gradients (loss, dW[l], db[l]) of the summed NLL scaled by 1/(B S)."""
    y, zs, hs = forward(X, W, b)
    loss, g = nll_grad(y, tgt)
    L = len(W)
    dW = [None] * L
    db = [None] * L
    dW[L - 1] = (g.T.astype(np.float64) @ hs[L - 1].astype(np.float64)).astype(np.float32)
    db[L - 1] = g.astype(np.float64).sum(0).astype(np.float32)
    for l in range(L - 2, -1, -1):
        dh = (g.astype(np.float64) @ bf16(W[l + 1]).astype(np.float64)).astype(np.float32)
        dz = bf16(dh * silu_grad(zs[l]))
        dW[l] = (dz.T.astype(np.float64) @ hs[l].astype(np.float64)).astype(np.float32)
        db[l] = dz.astype(np.float64).sum(0).astype(np.float32)
        g = dz
    return loss, dW, db, y
