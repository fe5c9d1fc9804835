"""CPU oracle for the cuTauLeaping hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package.  The product (``cutauleaping_b200``) never does.

ctypes bindings over ``libctl_oracle.so`` (built from ``ctl_oracle.c`` by the
Makefile next to this file).  The C code restates the reference routine
(``2phase_n-tau-leaping.cu`` PreCalculations 1568-2093, EventualSSASteps
2099-2273, LightweightSSA 2280-2454, helpers 1300-1562) under the canonical
arithmetic contract that the CUDA kernels reproduce bit for bit, plus an exact
FP64 Gillespie direct method.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# CTL_ORACLE_LIB selects another build of the same source (the sanitizer
# test loads one compiled with -fsanitize=address,undefined).
LIB_PATH = os.environ.get("CTL_ORACLE_LIB") or os.path.join(HERE, "libctl_oracle.so")

# Quirk switches (0 = reference behaviour); must match ctl_oracle.h.
FORCE_SSA = 1 << 0
Q1_OFF = 1 << 1
Q2_OFF = 1 << 2
Q3_OFF = 1 << 3
Q4_OFF = 1 << 4
Q5_OFF = 1 << 5
Q6_OFF = 1 << 6
Q9_OFF = 1 << 7
Q10_OFF = 1 << 8
ALL_QUIRKS_OFF = Q1_OFF | Q2_OFF | Q3_OFF | Q4_OFF | Q5_OFF | Q6_OFF | Q9_OFF | Q10_OFF

INFO_DTYPE = np.dtype([
    ("t_final", "<f8"), ("firings", "<u8"), ("status", "<u4"), ("steps", "<u4"),
    ("leaps", "<u4"), ("ssa_steps", "<u4"), ("rejections", "<u4"), ("pad", "<u4"),
])

_lib = None


def build(force: bool = False) -> str:
    """Compile libctl_oracle.so with the Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.ctlo_model_new.restype = P
        L.ctlo_model_new.argtypes = [C.c_int, C.c_int, P, P, P, C.c_int, P, C.c_int, P,
                                     C.c_float, C.c_uint32, C.c_double, C.c_uint32,
                                     C.c_uint32, C.c_uint64, C.c_uint32]
        L.ctlo_model_free.argtypes = [P]
        L.ctlo_model_hor.argtypes = [P, P, P]
        L.ctlo_simulate.argtypes = [P, C.c_uint32, P, P, P, P]
        L.ctlo_gillespie.argtypes = [P, C.c_uint32, P, P, P, P]
        L.ctlo_run_batch.argtypes = [P, C.c_int, C.c_uint32, P, P, P, P, C.c_int, C.c_int]
        L.ctlo_philox.argtypes = [P, P, P]
        L.ctlo_log.restype = C.c_double
        L.ctlo_log.argtypes = [C.c_double]
        L.ctlo_logf.restype = C.c_float
        L.ctlo_logf.argtypes = [C.c_float]
        L.ctlo_exp.restype = C.c_double
        L.ctlo_exp.argtypes = [C.c_double]
        L.ctlo_logfact.restype = C.c_double
        L.ctlo_logfact.argtypes = [C.c_double]
        L.ctlo_poisson.restype = C.c_uint32
        L.ctlo_poisson.argtypes = [C.c_double, C.c_uint64, C.c_uint32, C.c_uint32,
                                   C.c_uint32, C.c_uint32]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().ctlo_philox(_p(c), _p(k), _p(o))
    return o


def log(x: float) -> float:
    return lib().ctlo_log(float(x))


def logf(x: float) -> float:
    return lib().ctlo_logf(float(x))


def exp(x: float) -> float:
    return lib().ctlo_exp(float(x))


def logfact(k: float) -> float:
    return lib().ctlo_logfact(float(k))


def poisson(lam: float, seed: int, sim: int, step: int, attempt: int, r: int) -> int:
    return lib().ctlo_poisson(float(lam), seed, sim, step, attempt, r)


class OracleModel:
    """A reaction network plus run settings, held by the C oracle."""

    def __init__(self, left, right, feed, tvec, cs=None, *, eps=0.03, nc=10,
                 ssa_factor=10.0, ssa_steps=100, flags=0, seed=0, max_steps=0xFFFFFFFF):
        self.left = np.ascontiguousarray(left, dtype=np.int32)
        self.right = np.ascontiguousarray(right, dtype=np.int32)
        self.R, self.S = self.left.shape
        self.feed = np.ascontiguousarray(
            np.zeros(self.S) if feed is None else feed, dtype=np.int32)
        self.tvec = np.ascontiguousarray(tvec, dtype=np.float64)
        self.cs = np.ascontiguousarray(np.arange(self.S) if cs is None else cs, dtype=np.int32)
        self.ns, self.s_out = len(self.tvec), len(self.cs)
        self._h = lib().ctlo_model_new(self.S, self.R, _p(self.left), _p(self.right),
                                       _p(self.feed), self.ns, _p(self.tvec), self.s_out,
                                       _p(self.cs), eps, nc, ssa_factor, ssa_steps, flags,
                                       seed, max_steps)
        if not self._h:
            raise ValueError("oracle rejected the model")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.ctlo_model_free(h)
            self._h = None

    def hor(self):
        hor = np.zeros(self.S, np.uint8)
        hort = np.zeros(self.S, np.uint8)
        lib().ctlo_model_hor(self._h, _p(hor), _p(hort))
        return hor, hort

    def run(self, X0, c, *, sim_base=0, threads=None, mode=0):
        """Simulate n = len(X0) simulations; returns (samples [n][ns][s_out], info [n])."""
        X0 = np.ascontiguousarray(X0, dtype=np.int32).reshape(-1, self.S)
        c = np.ascontiguousarray(c, dtype=np.float32).reshape(-1, self.R)
        n = X0.shape[0]
        assert c.shape[0] == n
        out = np.zeros((n, self.ns, self.s_out), dtype=np.uint32)
        info = np.zeros(n, dtype=INFO_DTYPE)
        if threads is None:
            threads = os.cpu_count() or 1
        rc = lib().ctlo_run_batch(self._h, n, sim_base, _p(X0), _p(c), _p(out), _p(info),
                                  int(threads), int(mode))
        if rc:
            raise RuntimeError(f"oracle batch failed ({rc})")
        return out, info

    def gillespie(self, X0, c, *, sim_base=0, threads=None):
        return self.run(X0, c, sim_base=sim_base, threads=threads, mode=1)
