"""cutauleaping_b200 -- B200-native (sm_100a) drop-in for the simulation path of
aresio/cuTauLeaping.

The product is native: ``libctl.so`` (CUDA sweep + C++ host code, C ABI in
``include/ctl.h``) and the ``cutauleaping`` CLI with the reference's argv
contract (kernel.cu:74-436).  This module binds the C ABI through ctypes for
Python callers; it never falls back to a CPU implementation -- importing it
without the built library raises.

    import cutauleaping_b200 as ctl
    m = ctl.Model.load("schlogl_folder")          # left_side, right_side, ...
    X0, c = ctl.load_rows("schlogl_folder", m, offset=0, n=4096)
    samples, info = m.run(X0, c, seed=1)          # samples [n][ns][s_out]
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libctl.so")
CLI_PATH = os.path.join(HERE, "cutauleaping")

# ---- constants mirrored from include/ctl.h --------------------------------
OK, ERR_IO, ERR_PARSE, ERR_SHAPE, ERR_CUDA, ERR_OOM, ERR_STEP_LIMIT, ERR_TIMEOUT, ERR_ARG = range(9)
SIM_OK, SIM_STEP_LIMIT, SIM_OVERFLOW, SIM_ATTEMPT_LIMIT = range(4)
FORCE_SSA = 1 << 0
Q1_OFF, Q2_OFF, Q3_OFF, Q4_OFF, Q5_OFF, Q6_OFF, Q9_OFF, Q10_OFF = (1 << i for i in range(1, 9))
ALL_QUIRKS_OFF = Q1_OFF | Q2_OFF | Q3_OFF | Q4_OFF | Q5_OFF | Q6_OFF | Q9_OFF | Q10_OFF

INFO_DTYPE = np.dtype([
    ("t_final", "<f8"), ("firings", "<u8"), ("status", "<u4"), ("steps", "<u4"),
    ("leaps", "<u4"), ("ssa_steps", "<u4"), ("rejections", "<u4"), ("pad", "<u4"),
])

# Every symbol include/ctl.h declares (checked by the tests).
EXPORTS = [
    "ctl_status_str", "ctl_last_error", "ctl_last_error_detail", "ctl_model_load", "ctl_model_create", "ctl_model_free",
    "ctl_model_dims_get", "ctl_model_hor", "ctl_rows_load", "ctl_run_cfg_default", "ctl_run",
    "ctl_run_device", "ctl_run_device_noalloc", "ctl_launch_query", "ctl_autotune", "ctl_graph_create", "ctl_graph_create_multi", "ctl_graph_launch", "ctl_graph_free",
    "ctl_write_dynamics", "ctl_print_dynamics", "ctl_write_samples_binary", "ctl_write_run_report", "ctl_target_load", "ctl_target_free",
    "ctl_target_dims", "ctl_fitness", "ctl_fitness_device", "ctl_mlp_gemm", "ctl_mlp_nll_grad", "ctl_mlp_colsum",
    "ctl_mlp_adam", "ctl_mlp_pack_bytes", "ctl_mlp_pack", "ctl_mlp_screen", "ctl_mlp_wait_check", "ctl_run_device_sums",
    "ctl_fitness_sums_device", "ctl_fitness_run", "ctl_spec_source",
]


class RunCfg(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("eps", C.c_float), ("nc", C.c_uint32),
                ("ssa_factor", C.c_double), ("ssa_steps", C.c_uint32), ("flags", C.c_uint32),
                ("max_steps", C.c_uint32), ("sim_base", C.c_uint32), ("device", C.c_int32),
                ("group", C.c_int32), ("threads", C.c_int32), ("uniform_rates", C.c_int32),
                ("ssa_budget", C.c_int32), ("dec_budget", C.c_int32), ("min_blocks", C.c_int32),
                ("sched", C.c_int32), ("warp_sims", C.c_int32), ("spec", C.c_int32)]


class ModelDims(C.Structure):
    _fields_ = [("S", C.c_int32), ("R", C.c_int32), ("P", C.c_int32), ("ns", C.c_int32),
                ("s_out", C.c_int32), ("nnz_left", C.c_int32), ("nnz_var", C.c_int32),
                ("nnz_feared", C.c_int32), ("nnz_dep", C.c_int32), ("tmax", C.c_double)]


class LaunchInfo(C.Structure):
    _fields_ = [("group", C.c_int32), ("threads", C.c_int32), ("blocks", C.c_int32),
                ("slots_per_block", C.c_int32), ("smem_bytes", C.c_int32),
                ("regs_per_thread", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("sm_count", C.c_int32), ("min_blocks", C.c_int32), ("sched", C.c_int32),
                ("ssa_budget", C.c_int32), ("dec_budget", C.c_int32), ("warp_sims", C.c_int32),
                ("specialized", C.c_int32)]


class CtlError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        L = lib()
        msg = L.ctl_status_str(status).decode()
        detail = L.ctl_last_error().decode()
        self.detail = int(L.ctl_last_error_detail())
        super().__init__(f"{where}: {msg}" + (f": {detail}" if detail else ""))


_lib = None


def lib():
    """Load libctl.so; raises if the native library has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cutauleaping_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        st = C.c_int
        L.ctl_status_str.restype = C.c_char_p
        L.ctl_status_str.argtypes = [st]
        L.ctl_last_error.restype = C.c_char_p
        L.ctl_last_error_detail.restype = C.c_int32
        L.ctl_model_load.argtypes = [C.c_char_p, C.POINTER(P)]
        L.ctl_model_create.argtypes = [C.c_int32, C.c_int32, P, P, P, C.c_int32, P, C.c_int32, P,
                                       C.POINTER(P)]
        L.ctl_model_free.argtypes = [P]
        L.ctl_model_free.restype = None
        L.ctl_model_dims_get.argtypes = [P, C.POINTER(ModelDims)]
        L.ctl_model_hor.argtypes = [P, P, P]
        L.ctl_rows_load.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, P, P]
        L.ctl_run_cfg_default.argtypes = [C.POINTER(RunCfg)]
        L.ctl_run_cfg_default.restype = None
        L.ctl_run.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, P, P, P, P]
        L.ctl_run_device.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, P, P, P, P, P]
        L.ctl_launch_query.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, C.POINTER(LaunchInfo)]
        L.ctl_spec_source.argtypes = [P, C.c_int32, C.c_int32, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.ctl_run_device_noalloc.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, P, P, P, P, P]
        L.ctl_autotune.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, P, P, C.c_uint32, C.POINTER(LaunchInfo)]
        L.ctl_graph_create.argtypes = [P, C.POINTER(RunCfg), C.c_uint32, P, P, P, P, P, C.POINTER(P)]
        L.ctl_graph_create_multi.argtypes = [C.c_uint32, P, P, P, P, P, P, P, P, C.POINTER(P)]
        L.ctl_graph_launch.argtypes = [P, P]
        L.ctl_graph_free.argtypes = [P]
        L.ctl_graph_free.restype = None
        L.ctl_write_dynamics.argtypes = [P, C.c_char_p, C.c_uint32, P, C.c_uint32, C.c_int32]
        L.ctl_print_dynamics.argtypes = [P, C.c_uint32, P]
        L.ctl_write_samples_binary.argtypes = [P, C.c_char_p, C.c_uint32, P, C.c_uint32]
        L.ctl_write_run_report.argtypes = [P, C.c_char_p, C.c_uint32, P, C.c_double, P]
        L.ctl_target_load.argtypes = [C.c_char_p, P, C.c_uint32, C.c_uint32, C.POINTER(P)]
        L.ctl_target_free.argtypes = [P]
        L.ctl_target_free.restype = None
        L.ctl_target_dims.argtypes = [P, P, P, P, P]
        L.ctl_fitness.argtypes = [P, P, C.POINTER(RunCfg), P, P]
        L.ctl_fitness_device.argtypes = [P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_uint32, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(status: int, where: str):
    if status != OK:
        raise CtlError(status, where)


def run_cfg(*, seed=0, eps=0.03, nc=10, ssa_factor=10.0, ssa_steps=100, flags=0,
            max_steps=0xFFFFFFFF, sim_base=0, device=0, group=0, threads=0, uniform_rates=0,
            ssa_budget=0, dec_budget=0, min_blocks=0, sched=0, warp_sims=0, spec=0) -> RunCfg:
    cfg = RunCfg()
    lib().ctl_run_cfg_default(C.byref(cfg))
    cfg.seed, cfg.eps, cfg.nc, cfg.ssa_factor = seed, eps, nc, ssa_factor
    cfg.ssa_steps, cfg.flags, cfg.max_steps, cfg.sim_base = ssa_steps, flags, max_steps, sim_base
    cfg.device, cfg.group, cfg.threads = device, group, threads
    cfg.uniform_rates, cfg.ssa_budget, cfg.dec_budget = uniform_rates, ssa_budget, dec_budget
    cfg.min_blocks, cfg.sched, cfg.warp_sims, cfg.spec = min_blocks, sched, warp_sims, spec
    return cfg


class Model:
    """A reaction network and its sampling plan (opaque ctl_model handle)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        d = ModelDims()
        _check(lib().ctl_model_dims_get(self._h, C.byref(d)), "ctl_model_dims_get")
        self.S, self.R, self.P, self.ns, self.s_out = d.S, d.R, d.P, d.ns, d.s_out
        self.tmax = d.tmax
        self.dims = d

    @classmethod
    def load(cls, folder: str) -> "Model":
        h = C.c_void_p()
        _check(lib().ctl_model_load(os.fsencode(folder), C.byref(h)), "ctl_model_load")
        return cls(h.value)

    @classmethod
    def create(cls, left, right, feed, tvec, cs=None) -> "Model":
        left = np.ascontiguousarray(left, dtype=np.int32)
        right = np.ascontiguousarray(right, dtype=np.int32)
        R, S = left.shape
        feed_a = None if feed is None else np.ascontiguousarray(feed, dtype=np.int32)
        tvec = np.ascontiguousarray(tvec, dtype=np.float64)
        cs_a = None if cs is None else np.ascontiguousarray(cs, dtype=np.int32)
        h = C.c_void_p()
        _check(lib().ctl_model_create(S, R, _p(left), _p(right),
                                      None if feed_a is None else _p(feed_a), len(tvec), _p(tvec),
                                      0 if cs_a is None else len(cs_a),
                                      None if cs_a is None else _p(cs_a), C.byref(h)),
               "ctl_model_create")
        return cls(h.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ctl_model_free(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def hor(self):
        hor = np.zeros(self.S, np.uint8)
        hort = np.zeros(self.S, np.uint8)
        _check(lib().ctl_model_hor(self._h, _p(hor), _p(hort)), "ctl_model_hor")
        return hor, hort

    def run(self, X0, c, cfg: RunCfg | None = None, *, check=True, **kw):
        """Host-buffer sweep (ctl_run): returns (samples [n][ns][s_out] uint32, info [n])."""
        cfg = cfg if cfg is not None else run_cfg(**kw)
        X0 = np.ascontiguousarray(X0, dtype=np.int32).reshape(-1, self.S)
        c = np.ascontiguousarray(c, dtype=np.float32).reshape(-1, self.R)
        n = X0.shape[0]
        if c.shape[0] != n:
            raise ValueError("X0 and c must have the same number of rows")
        out = np.zeros((n, self.ns, self.s_out), dtype=np.uint32)
        info = np.zeros(n, dtype=INFO_DTYPE)
        st = lib().ctl_run(self._h, C.byref(cfg), n, _p(X0), _p(c), _p(out), _p(info))
        if st != OK and (check or st != ERR_STEP_LIMIT):
            raise CtlError(st, "ctl_run")
        return out, info

    def run_device(self, n, d_X0, d_c, d_out, d_info, stream=0, cfg: RunCfg | None = None, **kw):
        """Enqueue the sweep on device pointers (ints) and a raw cudaStream_t."""
        cfg = cfg if cfg is not None else run_cfg(**kw)
        _check(lib().ctl_run_device(self._h, C.byref(cfg), n, C.c_void_p(d_X0), C.c_void_p(d_c),
                                    C.c_void_p(d_out), C.c_void_p(d_info), C.c_void_p(stream)),
               "ctl_run_device")

    def spec_source(self, group: int, min_blocks: int = 3) -> str:
        """The CUDA source the library compiles with NVRTC for this network's
        shared-memory sweep (ctl_spec_source); no device work."""
        n = C.c_size_t()
        _check(lib().ctl_spec_source(self._h, group, min_blocks, None, 0, C.byref(n)), "ctl_spec_source")
        buf = C.create_string_buffer(n.value + 1)
        _check(lib().ctl_spec_source(self._h, group, min_blocks, buf, n.value + 1, C.byref(n)), "ctl_spec_source")
        return buf.value.decode()

    def launch_info(self, n, cfg: RunCfg | None = None, **kw) -> LaunchInfo:
        cfg = cfg if cfg is not None else run_cfg(**kw)
        li = LaunchInfo()
        _check(lib().ctl_launch_query(self._h, C.byref(cfg), n, C.byref(li)), "ctl_launch_query")
        return li

    def autotune(self, n, d_X0, d_c, sample=0, cfg: RunCfg | None = None, **kw) -> LaunchInfo:
        """Measure launch shapes on the first `sample` simulations (ctl_autotune)."""
        cfg = cfg if cfg is not None else run_cfg(**kw)
        li = LaunchInfo()
        _check(lib().ctl_autotune(self._h, C.byref(cfg), n, C.c_void_p(d_X0), C.c_void_p(d_c), sample,
                                  C.byref(li)), "ctl_autotune")
        return li

    def graph(self, n, d_X0, d_c, d_out, d_info, stream=0, cfg: RunCfg | None = None, **kw):
        cfg = cfg if cfg is not None else run_cfg(**kw)
        h = C.c_void_p()
        _check(lib().ctl_graph_create(self._h, C.byref(cfg), n, C.c_void_p(d_X0), C.c_void_p(d_c),
                                      C.c_void_p(d_out), C.c_void_p(d_info), C.c_void_p(stream),
                                      C.byref(h)), "ctl_graph_create")
        return Graph(h.value)

    def write_dynamics(self, path_prefix: str, samples, first_id=0, threads=0):
        samples = np.ascontiguousarray(samples, dtype=np.uint32)
        _check(lib().ctl_write_dynamics(self._h, os.fsencode(path_prefix), samples.shape[0],
                                        _p(samples), first_id, threads), "ctl_write_dynamics")

    def write_run_report(self, path: str, info, seconds: float, launch: "LaunchInfo | None" = None):
        """JSON run report for the records `info` of a run that took
        `seconds` (ctl_write_run_report)."""
        info = np.ascontiguousarray(info)
        if info.dtype != INFO_DTYPE:
            info = info.view(INFO_DTYPE).reshape(-1)
        _check(lib().ctl_write_run_report(self._h, os.fsencode(path), info.shape[0], _p(info), float(seconds),
                                          C.byref(launch) if launch is not None else None),
               "ctl_write_run_report")

    def write_samples_binary(self, path: str, samples, first_id=0):
        """The whole batch in one binary file (ctl_write_samples_binary);
        read it back with read_samples_binary."""
        samples = np.ascontiguousarray(samples, dtype=np.uint32)
        _check(lib().ctl_write_samples_binary(self._h, os.fsencode(path), samples.shape[0], _p(samples),
                                              first_id), "ctl_write_samples_binary")


def graph_multi(parts, stream=0) -> "Graph":
    """One CUDA graph running several batches as parallel branches
    (ctl_graph_create_multi).  parts: [(model, n, d_X0, d_c, d_out, d_info,
    cfg)] with device pointers as ints; each model at most once."""
    k = len(parts)
    models = (C.c_void_p * k)(*[p[0].handle.value for p in parts])
    cfgs = (RunCfg * k)(*[p[6] for p in parts])
    ns = (C.c_uint32 * k)(*[p[1] for p in parts])
    ptr = lambda i: (C.c_void_p * k)(*[p[i] for p in parts])
    h = C.c_void_p()
    _check(lib().ctl_graph_create_multi(k, models, cfgs, ns, ptr(2), ptr(3), ptr(4), ptr(5), C.c_void_p(stream),
                                        C.byref(h)), "ctl_graph_create_multi")
    return Graph(h.value)


class Graph:
    """A captured sweep (ctl_graph); replay with launch()."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    def launch(self, stream=0):
        _check(lib().ctl_graph_launch(self._h, C.c_void_p(stream)), "ctl_graph_launch")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ctl_graph_free(h)
            self._h = None


SAMPLES_MAGIC = b"CTLSAMP1"


def read_samples_binary(path: str, mmap: bool = True):
    """Read a file written by ctl_write_samples_binary (or the CLI with
    CTL_BINARY_OUTPUT=1): returns dict(t [ns] float64, species [s_out],
    first_id, samples [n][ns][s_out] uint32 -- memory-mapped unless mmap is
    False).  Raises ValueError on a file of another format or a short file."""
    with open(path, "rb") as f:
        head = f.read(24)
        if len(head) < 24 or head[:8] != SAMPLES_MAGIC:
            raise ValueError(f"{path}: not a sample file (magic {head[:8]!r})")
        n, ns, s_out, first_id = np.frombuffer(head, dtype="<u4", offset=8, count=4).tolist()
        t = np.frombuffer(f.read(8 * ns), dtype="<f8")
        species = np.frombuffer(f.read(4 * s_out), dtype="<u4")
        if t.size != ns or species.size != s_out:
            raise ValueError(f"{path}: truncated header")
    data_off = (24 + 8 * ns + 4 * s_out + 15) // 16 * 16
    need = data_off + 4 * n * ns * s_out
    if os.path.getsize(path) != need:
        raise ValueError(f"{path}: {os.path.getsize(path)} bytes, the header announces {need}")
    shape = (n, ns, s_out)
    if mmap and n * ns * s_out:
        samples = np.memmap(path, dtype="<u4", mode="r", offset=data_off, shape=shape)
    else:
        samples = np.fromfile(path, dtype="<u4", count=n * ns * s_out, offset=data_off).reshape(shape)
    return {"t": t.copy(), "species": species.copy(), "first_id": first_id, "samples": samples}


def load_rows(folder: str, model: Model, offset: int, n: int):
    """Rows [offset, offset+n) of MX_0 and c_matrix (ctl_rows_load)."""
    X0 = np.zeros((n, model.S), dtype=np.int32)
    c = np.zeros((n, model.R), dtype=np.float32)
    _check(lib().ctl_rows_load(os.fsencode(folder), model.S, model.R, offset, n, _p(X0), _p(c)),
           "ctl_rows_load")
    return X0, c


class Target:
    """Fitness targets (ctl_target): ts_rep, p_rep, ts_numtgt, tts_vector, ts_matrix."""

    def __init__(self, folder: str, model: Model, threads: int, blocks: int):
        h = C.c_void_p()
        _check(lib().ctl_target_load(os.fsencode(folder), model.handle, threads, blocks, C.byref(h)),
               "ctl_target_load")
        self._h = h
        self.threads, self.blocks = threads, blocks
        v = [C.c_uint32() for _ in range(4)]
        _check(lib().ctl_target_dims(h, *[C.byref(x) for x in v]), "ctl_target_dims")
        self.repetitions, self.p_rep, self.target_quantities, self.experiments = (x.value for x in v)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.ctl_target_free(h)
            self._h = None

    def fitness(self, model: Model, samples, cfg: RunCfg | None = None, **kw):
        cfg = cfg if cfg is not None else run_cfg(**kw)
        samples = np.ascontiguousarray(samples, dtype=np.uint32)
        out = np.zeros(self.threads * self.blocks, dtype=np.float64)
        _check(lib().ctl_fitness(model.handle, self._h, C.byref(cfg), _p(samples), _p(out)),
               "ctl_fitness")
        return out
