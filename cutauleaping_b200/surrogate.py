"""Learned surrogate for the fitness mode (parameter estimation).

The reference computes the fitness of every candidate parameter set by full
simulation (kernel.cu:365-423, calculateFitness 2phase_n-tau-leaping.cu:
3324-3408).  Here a small MLP, trained on trajectories the simulator itself
produces, screens candidates first; every retained candidate is re-simulated
with the plain method, which also measures the surrogate's error.

Network: x = (8 scaled log rate constants, scaled t) -> 256 -> 256 -> 256 ->
256 -> 2*S (per-species mean and log-variance of the standardised counts),
SiLU, BF16 weights and activations, FP32 accumulation and master weights,
Gaussian negative log-likelihood, Adam.  Every matrix product of training
runs in the project's own tcgen05 kernel (ctl_mlp_gemm); the loss gradient,
bias gradients and Adam are the project's own kernels too.  Screening runs
the whole network and the fitness in one fused tcgen05 kernel
(ctl_mlp_screen, `screen`).  PyTorch only provides device memory.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import CtlError, OK, lib

EPI_ATOMIC_F32, EPI_BIAS_SILU, EPI_BIAS, EPI_SILU_GRAD, EPI_F32 = range(5)
IN_PAD = 64      # 9 inputs padded to one K tile
HIDDEN = 256
LAYERS = 4       # hidden layers of width 256


class GemmDesc(C.Structure):
    _fields_ = [("A", C.c_void_p), ("B", C.c_void_p), ("lda", C.c_int32), ("ldb", C.c_int32),
                ("M", C.c_int32), ("N", C.c_int32), ("K", C.c_int32), ("epilogue", C.c_int32),
                ("splits", C.c_int32), ("bias", C.c_void_p), ("z_in", C.c_void_p), ("ldz", C.c_int32),
                ("out_f32", C.c_void_p), ("ldo", C.c_int32), ("out_bf", C.c_void_p), ("ldob", C.c_int32),
                ("out_bfT", C.c_void_p), ("ldobT", C.c_int32), ("err", C.c_void_p)]


class ScreenDesc(C.Structure):
    _fields_ = [("theta", C.c_void_p), ("n_par", C.c_int32), ("n_cand", C.c_uint32), ("tvec", C.c_void_p),
                ("ns", C.c_uint32), ("t_end", C.c_float), ("log_lo", C.c_void_p), ("log_hi", C.c_void_p),
                ("y_mean", C.c_void_p), ("y_std", C.c_void_p), ("S", C.c_int32), ("out_w", C.c_int32),
                ("target", C.c_void_p), ("wpack", C.c_void_p), ("bias", C.c_void_p), ("fitness", C.c_void_p),
                ("err", C.c_void_p)]


def _bind():
    L = lib()
    if not getattr(L, "_mlp_bound", False):
        P = C.c_void_p
        L.ctl_mlp_pack_bytes.argtypes = [C.c_int32]
        L.ctl_mlp_pack_bytes.restype = C.c_size_t
        L.ctl_mlp_pack.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_int32), C.c_int32, P, P]
        L.ctl_mlp_screen.argtypes = [C.POINTER(ScreenDesc), P]
        L.ctl_mlp_gemm.argtypes = [C.POINTER(GemmDesc), P]
        L.ctl_mlp_nll_grad.argtypes = [P, C.c_int32, P, C.c_int32, C.c_int32, P, C.c_int32, P, C.c_int32, P, P]
        L.ctl_mlp_colsum.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, P, P]
        L.ctl_mlp_adam.argtypes = [P, P, P, P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float,
                                   C.c_float, C.c_int32, C.c_float, P, P, P]
        L._mlp_bound = True
    return L


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def gemm(A, B, *, epilogue, out_f32=None, out_bf=None, out_bfT=None, bias=None, z_in=None,
         splits=1, err=None):
    """C = A . B^T (A [M][K], B [N][K], BF16 torch tensors) on the tcgen05 kernel."""
    L = _bind()
    M, K = A.shape
    N, K2 = B.shape
    assert K == K2
    d = GemmDesc(_ptr(A), _ptr(B), A.stride(0), B.stride(0), M, N, K, epilogue, splits,
                 _ptr(bias), _ptr(z_in), 0 if z_in is None else z_in.stride(0),
                 _ptr(out_f32), 0 if out_f32 is None else out_f32.stride(0),
                 _ptr(out_bf), 0 if out_bf is None else out_bf.stride(0),
                 _ptr(out_bfT), 0 if out_bfT is None else out_bfT.stride(0), _ptr(err))
    st = L.ctl_mlp_gemm(C.byref(d), _stream())
    if st != OK:
        raise CtlError(st, "ctl_mlp_gemm")


@dataclass
class Scaling:
    """Input and output scaling of the surrogate."""
    log_lo: np.ndarray      # [8] log of the prior box low end
    log_hi: np.ndarray      # [8]
    t_end: float
    y_mean: np.ndarray      # [S] per-species mean count
    y_std: np.ndarray       # [S]


def make_inputs(theta_log, t, sc: Scaling, torch_mod):
    """X [n][64] BF16: scaled log rate constants in [-1, 1], scaled time, zeros."""
    torch = torch_mod
    n = theta_log.shape[0]
    X = torch.zeros((n, IN_PAD), dtype=torch.float32, device="cuda")
    lo = torch.as_tensor(sc.log_lo, dtype=torch.float32, device="cuda")
    hi = torch.as_tensor(sc.log_hi, dtype=torch.float32, device="cuda")
    X[:, :8] = 2.0 * (theta_log - lo) / (hi - lo) - 1.0
    X[:, 8] = 2.0 * t / sc.t_end - 1.0
    return X.to(torch.bfloat16)


class MLP:
    """9 -> 256 x 4 -> 2S surrogate with its own tcgen05 forward/backward."""

    def __init__(self, S: int, seed: int = 0):
        import torch
        self.torch = torch
        self.S = S
        if 2 * S > 128:
            raise ValueError("the surrogate predicts at most 64 species")
        self.out_w = max(64, (2 * S + 63) // 64 * 64)  # output layer padded to a K tile
        self.dims = [IN_PAD] + [HIDDEN] * LAYERS + [self.out_w]
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W, self.b, self.Wb, self.WbT, self.m, self.v, self.mb, self.vb = ([] for _ in range(8))
        for l in range(len(self.dims) - 1):
            fan_in, fan_out = (9 if l == 0 else self.dims[l]), self.dims[l + 1]
            w = torch.zeros(fan_out, self.dims[l])
            live = 2 * S if l == len(self.dims) - 2 else fan_out  # padded outputs stay zero
            w[:live, :fan_in] = torch.randn(live, fan_in, generator=g) * math.sqrt(1.0 / fan_in)
            if l == len(self.dims) - 2:
                w *= 0.1
            w = w.cuda()
            self.W.append(w)
            self.b.append(torch.zeros(fan_out, device="cuda"))
            self.Wb.append(w.to(torch.bfloat16).contiguous())
            self.WbT.append(w.t().contiguous().to(torch.bfloat16))
            self.m.append(torch.zeros_like(w))
            self.v.append(torch.zeros_like(w))
            self.mb.append(torch.zeros(fan_out, device="cuda"))
            self.vb.append(torch.zeros(fan_out, device="cuda"))
        self.step_count = 0   # Adam's bias-correction step
        self.version = 0      # changes with every weight update (keys the packed copy)
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self._bufs = {}

    # -- buffers ---------------------------------------------------------------
    def _buf(self, name, shape, dtype):
        t = self._bufs.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = self.torch.empty(shape, dtype=dtype, device="cuda")
            self._bufs[name] = t
        return t

    def forward(self, X, keep=True):
        """X [B][64] BF16 (B % 128 == 0) -> y [B][2S] FP32."""
        torch = self.torch
        Bn = X.shape[0]
        h = X
        self.h = [X]
        self.z = []
        self.hT = []
        for l in range(LAYERS):
            z = self._buf(f"z{l}", (Bn, HIDDEN), torch.float32)
            hn = self._buf(f"h{l}", (Bn, HIDDEN), torch.bfloat16)
            hT = self._buf(f"hT{l}", (HIDDEN, Bn), torch.bfloat16) if keep else None
            gemm(h, self.Wb[l], epilogue=EPI_BIAS_SILU, out_f32=z, out_bf=hn, out_bfT=hT,
                 bias=self.b[l], err=self.err)
            self.z.append(z)
            self.h.append(hn)
            self.hT.append(hT)
            h = hn
        y = self._buf("y", (Bn, self.out_w), torch.float32)
        gemm(h, self.Wb[LAYERS], epilogue=EPI_BIAS, out_f32=y, bias=self.b[LAYERS], err=self.err)
        return y

    def backward(self, y, target):
        """Gaussian NLL of y = [mu | log var] against target [B][S]; returns
        (loss sum, gradients dW[l], db[l])."""
        torch = self.torch
        L = _bind()
        Bn, S = target.shape
        dy = self._buf("dy", (Bn, self.out_w), torch.bfloat16)
        dy.zero_()
        dyT = self._buf("dyT", (128, Bn), torch.bfloat16)
        dyT.zero_()
        loss = torch.zeros(1, device="cuda")
        st = L.ctl_mlp_nll_grad(_ptr(y), y.stride(0), _ptr(target), Bn, S, _ptr(dy), dy.stride(0), _ptr(dyT), Bn,
                                _ptr(loss), _stream())
        if st != OK:
            raise CtlError(st, "ctl_mlp_nll_grad")
        XT = self._buf("XT", (IN_PAD, Bn), torch.bfloat16)
        XT.copy_(self.h[0].t())
        dW = [torch.zeros_like(w) if l < LAYERS else torch.zeros(128, HIDDEN, device="cuda")
              for l, w in enumerate(self.W)]
        db = [torch.zeros_like(b) for b in self.b]
        splits = max(1, min(64, Bn // 512))
        # output layer
        gemm(dyT, self.hT[LAYERS - 1], epilogue=EPI_ATOMIC_F32, out_f32=dW[LAYERS], splits=splits, err=self.err)
        L.ctl_mlp_colsum(_ptr(dy), Bn, self.out_w, self.out_w, _ptr(db[LAYERS]), _stream())
        g = dy
        for l in range(LAYERS - 1, -1, -1):
            dz = self._buf(f"dz{l}", (Bn, HIDDEN), torch.bfloat16)
            dzT = self._buf(f"dzT{l}", (HIDDEN, Bn), torch.bfloat16)
            gemm(g, self.WbT[l + 1], epilogue=EPI_SILU_GRAD, z_in=self.z[l], out_bf=dz, out_bfT=dzT, err=self.err)
            prevT = self.hT[l - 1] if l > 0 else XT
            gemm(dzT, prevT, epilogue=EPI_ATOMIC_F32, out_f32=dW[l], splits=splits, err=self.err)
            L.ctl_mlp_colsum(_ptr(dz), Bn, HIDDEN, HIDDEN, _ptr(db[l]), _stream())
            g = dz
        dW[LAYERS] = dW[LAYERS][: self.out_w].contiguous()
        return loss, dW, db

    def adam(self, dW, db, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.0):
        L = _bind()
        self.step_count += 1
        self.version += 1
        for l in range(len(self.W)):
            rows, cols = self.W[l].shape
            st = L.ctl_mlp_adam(_ptr(self.W[l]), _ptr(dW[l]), _ptr(self.m[l]), _ptr(self.v[l]), rows, cols,
                                lr, beta1, beta2, eps, self.step_count, wd, _ptr(self.Wb[l]),
                                _ptr(self.WbT[l]), _stream())
            if st != OK:
                raise CtlError(st, "ctl_mlp_adam")
            st = L.ctl_mlp_adam(_ptr(self.b[l]), _ptr(db[l]), _ptr(self.mb[l]), _ptr(self.vb[l]), 1, rows,
                                lr, beta1, beta2, eps, self.step_count, 0.0, None, None, _stream())
            if st != OK:
                raise CtlError(st, "ctl_mlp_adam")

    def packed(self):
        """Weights in the screening kernel's streaming layout and the
        concatenated biases; rebuilt after every Adam step."""
        torch = self.torch
        if getattr(self, "_packed_at", None) != self.version:
            L = _bind()
            wp = torch.empty(L.ctl_mlp_pack_bytes(self.out_w) // 2, dtype=torch.bfloat16, device="cuda")
            ptrs = (C.c_void_p * 5)(*[w.data_ptr() for w in self.Wb])
            lds = (C.c_int32 * 5)(*[w.stride(0) for w in self.Wb])
            st = L.ctl_mlp_pack(ptrs, lds, self.out_w, _ptr(wp), _stream())
            if st != OK:
                raise CtlError(st, "ctl_mlp_pack")
            self._wpack = wp
            self._bias = torch.cat(self.b).contiguous()
            self._packed_at = self.version
        return self._wpack, self._bias

    # -- optimiser state ---------------------------------------------------------
    _STATE = ("W", "b", "Wb", "WbT", "m", "v", "mb", "vb")

    def state(self):
        """A copy of the weights and the optimiser state."""
        st = {k: [t.clone() for t in getattr(self, k)] for k in self._STATE}
        st["step_count"] = self.step_count
        return st

    def load_state(self, st):
        for k in self._STATE:
            for dst, src in zip(getattr(self, k), st[k]):
                dst.copy_(src)
        self.step_count = st["step_count"]
        self.version += 1

    def reset_optimizer(self):
        """Fresh Adam moments (and bias correction) for a new training phase."""
        for k in ("m", "v", "mb", "vb"):
            for t in getattr(self, k):
                t.zero_()
        self.step_count = 0

    def check_error_flag(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("tcgen05 GEMM reported a bounded-wait timeout")

    def state_numpy(self):
        return ([w.cpu().numpy() for w in self.W], [b.cpu().numpy() for b in self.b])


def screen(net: MLP, theta_log, tvec, target, sc: Scaling):
    """Fitness of each candidate from the surrogate's ensemble mean, in one
    fused kernel (ctl_mlp_screen): theta_log [n][n_par] FP32 device tensor,
    tvec [ns], target [ns][S]; returns a FP64 device tensor [n]."""
    torch = net.torch
    L = _bind()
    dev = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float32, device="cuda").contiguous()
    theta = theta_log.to(torch.float32).contiguous()
    n, n_par = theta.shape
    tv, tg = dev(tvec), dev(target)
    lo, hi, ym, ys = dev(sc.log_lo), dev(sc.log_hi), dev(sc.y_mean), dev(sc.y_std)
    wp, bias = net.packed()
    fit = torch.empty(n, dtype=torch.float64, device="cuda")
    d = ScreenDesc(_ptr(theta), n_par, n, _ptr(tv), tv.shape[0], float(sc.t_end), _ptr(lo), _ptr(hi), _ptr(ym),
                   _ptr(ys), net.S, net.out_w, _ptr(tg), _ptr(wp), _ptr(bias), _ptr(fit), _ptr(net.err))
    st = L.ctl_mlp_screen(C.byref(d), _stream())
    if st != OK:
        raise CtlError(st, "ctl_mlp_screen")
    return fit
