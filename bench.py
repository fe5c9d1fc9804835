"""Benchmark: simulations/s (and reaction firings/s) of the tau-leaping sweep.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--config 2]

Workload (default, config 2): the synthetic mass-action network -- 64
species, 128 reactions of order 0-2 (generator seed 0), rate constants
log-uniform in [1e-4, 1], initial counts log-uniform in [10, 1e4] -- for
65,536 simulations per GPU, t_end = 10, 200 samples, eps = 0.03.  One step =
one complete sweep (every simulation from t = 0 to t_end), launched as one
CUDA graph (work-queue reset + persistent kernel).

  value     sims/s with inputs resident in HBM, CUDA-event time per step on the
            launching stream, L2 flushed (256 MB write) between steps, max over
            ranks.
  e2e       the same metric through the C ABI call a user makes (ctl_run) with
            pinned host buffers: H2D of X0/c, the sweep, D2H of all samples and
            per-simulation records, timed on the host around the call.
  io        output files timed apart from the sweep (rank 0, up to 4,096
            simulations' samples): the reference's text file per simulation
            against the one-file binary dump, seconds and bytes per simulation.
  --impl reference
            the reference routine on the host cores: the C restatement in
            oracle/ (the reference has no CPU implementation of its own), all
            host threads, a bounded sample of the same workload per step.

Multi-GPU (torchrun): every rank simulates its own 65,536 simulations
(disjoint Philox streams via sim_base), no collective on the data path;
value = all simulations / max-over-ranks time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sims/sec & reaction firings/sec on 1 B200 vs host build; surrogate-screened fits/sec"


def workload(config: int, n: int | None = None):
    """[(network, description)] segments of one benchmark step."""
    from cutauleaping_b200 import inputs
    if config == 1:
        net = inputs.schlogl(n or 4096)
        return [(net, f"Schlogl bistable model (schlogl.xml), {net.n} simulations, t_end=5, "
                      f"100 samples, eps=0.03, SSA factor 10, n_c=10")]
    if config == 3:
        half = (n or 1 << 20) // 2
        a = inputs.schlogl(half)
        a.c = a.c * np.exp(0.5 * np.random.default_rng(30).standard_normal(a.c.shape))
        b = inputs.synthetic(32, 64, half, seed=3, t_end=10.0, samples=200, perturb_sigma=0.5,
                             perturb_seed=31)
        return [(a, f"uneven batch part 1: Schlogl, {half} simulations with rates x exp(0.5 z)"),
                (b, f"uneven batch part 2: synthetic 32x64 (generator seed 3), {half} simulations "
                    f"with rates x exp(0.5 z), t_end=10, 200 samples")]
    if config == 4:
        net = inputs.synthetic(512, 1024, n or 16384, seed=0, t_end=20.0, samples=500,
                               c_range=(1e-5, 1e-1), x0_range=(1, 100000))
        return [(net, f"large sparse network 512 species x 1024 reactions (<= 4 nonzeros per "
                      f"reaction, generator seed 0), {net.n} simulations, t_end=20, 500 samples")]
    net = inputs.synthetic(64, 128, n or 65536, seed=0, t_end=10.0, samples=200)
    return [(net, f"synthetic mass-action network 64 species x 128 reactions (order 0-2, generator "
                  f"seed 0), {net.n} simulations, t_end=10, 200 samples, eps=0.03")]


def op_count(net, info):
    """Algorithmic 32-bit-op count of the sweep under a fixed convention:
    SSA step 6R + 2 nnz_F/R + 60; leap attempt 44R + 4 nnz_V + 8S + 2 nnz_F + 60;
    SSA hand-off decision 4R + 4 nnz_V + 8S."""
    S, R = net.S, net.R
    V = net.right - net.left
    F = V * (1 - net.feed[None, :])
    nnz_v, nnz_f = int((V != 0).sum()), int((F != 0).sum())
    w_ssa = 6 * R + 2 * nnz_f / R + 60
    w_leap = 44 * R + 4 * nnz_v + 8 * S + 2 * nnz_f + 60
    w_hand = 4 * R + 4 * nnz_v + 8 * S
    ssa = info["ssa_steps"].astype(np.float64)
    att = info["leaps"].astype(np.float64) + info["rejections"]
    hand = np.maximum(info["steps"].astype(np.float64) - ssa - info["leaps"], 0)
    return float((ssa * w_ssa + att * w_leap + hand * w_hand).sum())


def algorithmic_bytes(net):
    """HBM bytes one simulation must move: X0 (4S) + c (4R) + samples
    (4 ns s_out) + its 40-byte record."""
    so = net.S if net.cs is None else len(net.cs)
    return 4 * net.S + 4 * net.R + 4 * len(net.tvec) * so + 40


def io_timing(model, samples, threads: int = 0):
    """Output-file cost, timed apart from the sweep: the reference's text file
    per simulation (ctl_write_dynamics, WriteDynamics2's format) and the
    one-file binary dump (ctl_write_samples_binary) for `samples`
    [n][ns][s_out], written to a temporary folder that is removed after.
    Returns seconds per simulation for each, or the error when the host
    cannot write."""
    import shutil
    import tempfile
    n = int(samples.shape[0])
    d = tempfile.mkdtemp(prefix="ctl_io_")
    try:
        t0 = time.perf_counter()
        model.write_dynamics(os.path.join(d, "pref"), samples, threads=threads)
        t1 = time.perf_counter()
        model.write_samples_binary(os.path.join(d, "batch.ctlbin"), samples)
        t2 = time.perf_counter()
        text_bytes = sum(e.stat().st_size for e in os.scandir(d) if e.name.startswith("pref_"))
        return {"sample_sims": n, "threads": threads or os.cpu_count(),
                "text_s_per_sim": (t1 - t0) / n, "binary_s_per_sim": (t2 - t1) / n,
                "text_bytes_per_sim": text_bytes / n,
                "binary_bytes_per_sim": os.path.getsize(os.path.join(d, "batch.ctlbin")) / n,
                "folder": "temporary folder on the host's default temp file system"}
    except Exception as e:  # a full or read-only disk must not end the benchmark
        return {"error": f"{type(e).__name__}: {e}"}
    finally:
        shutil.rmtree(d, ignore_errors=True)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a moment to print its first row; a timed region
            # shorter than that (config 1: 5 x 13 ms) would have no sample at
            # all, so the region starts once the first row (taken under the
            # warm-up steps' load) is in
            t0 = time.time()
            while not self.rows and self.proc.poll() is None and time.time() - t0 < 3.0:
                time.sleep(0.005)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_reference(net, desc, steps, warmup, sample_s=10.0, threads=None, flags=0):
    """The reference routine on the host: oracle port, all host threads,
    bounded samples of the same workload.  Returns (sims/s, firings/s, meta)."""
    import oracle
    threads = threads or os.cpu_count() or 1
    m = oracle.OracleModel(net.left, net.right, net.feed, net.tvec, net.cs, seed=1, flags=flags)
    c32 = net.c.astype(np.float32)
    # size the sample so that one step takes about `sample_s` seconds
    k = min(net.n, max(threads, 64))
    t0 = time.perf_counter()
    m.run(net.X0[:k], c32[:k], threads=threads)
    per = (time.perf_counter() - t0) / k
    k = int(min(net.n, max(threads, sample_s / max(per, 1e-9))))
    vals, fvals = [], []
    for i in range(warmup + steps):
        lo = (i * k) % max(1, net.n - k + 1)
        t0 = time.perf_counter()
        _, info = m.run(net.X0[lo:lo + k], c32[lo:lo + k], sim_base=lo, threads=threads)
        dt = time.perf_counter() - t0
        if i >= warmup:
            vals.append(k / dt)
            fvals.append(float(info["firings"].sum()) / dt)
    return float(np.mean(vals)), float(np.mean(fvals)), {
        "cores": threads, "k": k, "sample": f"{k} of the {net.n} simulations per step ({desc.split(',')[0]})"}


def cpu_reference_segments(segs, steps, warmup, flags=0):
    """CPU port over every segment: sims/s of the whole step = total sims /
    sum of per-segment times (each measured on a bounded sample)."""
    tot_n, tot_t, tot_f, meta = 0, 0.0, 0.0, None
    budget = 10.0 / len(segs)
    samples, sample_ms = [], 0.0
    for net, desc in segs:
        v, fv, meta = cpu_reference(net, desc, steps, warmup, sample_s=budget, flags=flags)
        tot_n += net.n
        tot_t += net.n / v
        tot_f += fv * (net.n / v)
        samples.append(meta["sample"])
        sample_ms += 1e3 * meta["k"] / v
    return tot_n / tot_t, tot_f / tot_t, {"cores": meta["cores"], "sample": "; ".join(samples),
                                          "sample_ms": sample_ms}


def measured_peaks():
    """(peaks, source): the driver-measured peaks of this pool's B200s, or the
    earlier pool measurement (6,650 GB/s copy, 1,590 TFLOP/s bf16 burst) when
    the file is absent."""
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def screen_roofline(p, net, sc, n_cand):
    """Tensor roofline of the fused screening kernel (ctl_mlp_screen): n_cand
    candidates x ns instants rows, 2 * (64*256 + 3*256*256 + 256*out_w)
    FLOPs per row, CUDA events on the launching stream over 10 launches after
    3 warm-ups; peak = the measured burst BF16 GEMM rate."""
    import torch
    from cutauleaping_b200 import surrogate as sg
    rng = np.random.default_rng(12)
    th = torch.as_tensor(rng.uniform(p.log_lo, p.log_hi, size=(n_cand, len(p.unknown))), dtype=torch.float32,
                         device="cuda")
    tgt = p.target.astype(np.float32)
    for _ in range(3):
        sg.screen(net, th, p.tvec, tgt, sc)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    reps = 10
    for _ in range(reps):
        sg.screen(net, th, p.tvec, tgt, sc)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flops = float(n_cand * len(p.tvec)) * 2.0 * (64 * 256 + 3 * 256 * 256 + 256 * net.out_w)
    peaks, src = measured_peaks()
    peak = float(peaks.get("bf16_tflops", 1590.0))
    ach = flops / (ms * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": "screen_kernel (fused 5-layer MLP + fitness)", "achieved": ach,
            "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "traffic": None,
            "launch_ms": ms, "rows_per_launch": n_cand * len(p.tvec),
            "peak_source": f"MEASURED_PEAKS.json bf16_tflops ({src}, burst)" if src == "measured"
            else "fallback: 1,590 TFLOP/s bf16 burst (earlier pool measurement)"}


def bench_screen(a):
    """The fused screening kernel alone (config 5's tensor-core part): a
    briefly trained surrogate of the config-5 network scores 200,000
    candidates x 50 instants per launch; prints its roofline line."""
    import torch
    from cutauleaping_b200 import fitsearch as fs
    p = fs.make_problem(n_rep=8, samples=50, t_end=5.0)
    theta, traj = fs.training_data(p, 1 << 14)
    net, sc = fs.train_surrogate(p, theta, traj, epochs=1, batch=8192)
    torch.cuda.synchronize()
    r = screen_roofline(p, net, sc, n_cand=200_000)
    net.check_error_flag()
    print(json.dumps({"metric": "screened candidate-instants/s (fused surrogate screening kernel)",
                      "value": r["rows_per_launch"] / (r["launch_ms"] * 1e-3), "unit": "rows/s",
                      "higher_is_better": True, "n_gpus": 1, "dtype": "bf16 (fp32 accumulate)",
                      "data": "synthetic", "config": {"workload": "screening of 200,000 candidates x 50 instants, "
                                                                  "9 -> 256 x 4 -> 64 MLP + fitness"},
                      "roofline": r, "gpu_launches": 10}), flush=True)


def bench_gemm(a):
    """The surrogate's training GEMM alone (ctl_mlp_gemm, tcgen05): the
    hidden-layer forward product of a 16,384-row training batch (M = 16384,
    N = K = 256, bias + SiLU epilogue writing FP32 and BF16) and its weight
    gradient (M = N = 256, K = 16384, split-K 32 as training takes it:
    batch / 512, at most 64; FP32 atomic epilogue); 2MNK
    FLOPs per launch, CUDA events on the launching stream over 20 launches
    after 5 warm-ups; peak = the measured burst BF16 GEMM rate."""
    import torch
    from cutauleaping_b200 import surrogate as sg
    g = torch.Generator(device="cuda").manual_seed(3)
    B, W = 16384, 256
    X = torch.randn(B, W, device="cuda", generator=g).to(torch.bfloat16)
    Wt = (torch.randn(W, W, device="cuda", generator=g) / 16).to(torch.bfloat16)
    bias = torch.zeros(W, device="cuda")
    z = torch.empty(B, W, device="cuda")
    h = torch.empty(B, W, dtype=torch.bfloat16, device="cuda")
    XT = X.t().contiguous()
    dW = torch.zeros(W, W, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    peaks, src = measured_peaks()
    peak = float(peaks.get("bf16_tflops", 1590.0))
    shapes = {
        "forward (M=16384, N=256, K=256, bias+SiLU)": (lambda: sg.gemm(X, Wt, epilogue=sg.EPI_BIAS_SILU, out_f32=z,
                                                                      out_bf=h, bias=bias, err=err), B * W * W),
        "weight gradient (M=256, N=256, K=16384, split-K 32)": (lambda: sg.gemm(XT, XT, epilogue=sg.EPI_ATOMIC_F32,
                                                                               out_f32=dW, splits=32, err=err), W * W * B),
    }
    out = {}
    for name, (fn, mnk) in shapes.items():
        for _ in range(5):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 20
        ach = 2.0 * mnk / (ms * 1e-3) / 1e12
        out[name] = {"launch_ms": ms, "achieved": ach, "frac": ach / peak}
    if int(err.item()) != 0:
        raise RuntimeError("GEMM reported a bounded-wait timeout")
    fwd = out["forward (M=16384, N=256, K=256, bias+SiLU)"]
    print(json.dumps({"metric": "training GEMM TFLOP/s (tcgen05, surrogate training shapes)",
                      "value": fwd["achieved"], "unit": "TFLOP/s", "higher_is_better": True, "n_gpus": 1,
                      "dtype": "bf16 (fp32 accumulate)", "data": "synthetic",
                      "config": {"workload": "surrogate training GEMMs, 16,384-row batch, width 256"},
                      "roofline": {"bound": "tensor", "achieved": fwd["achieved"], "peak": peak, "unit": "TFLOP/s",
                                   "frac": fwd["frac"], "traffic": None,
                                   "peak_source": f"MEASURED_PEAKS.json bf16_tflops ({src}, burst)"},
                      "shapes": out, "gpu_launches": 50}), flush=True)


def bench_config5(a):
    """Surrogate-screened parameter estimation against plain-simulator search.

    Both searches run the same cross-entropy method (cutauleaping_b200.fitsearch)
    until their best true fitness is within 2% of the fitness of the true
    parameters (the attainable floor at this replicate count), or a generation
    cap.  The surrogate search pays for its training data and training inside
    its wall time, and after every generation fine-tunes the network on 8 of
    the trajectories it just simulated per candidate for half of them (half
    of each batch replayed from the original training data), keeping the
    fine-tuned weights only if the surrogate's error on the other half's
    simulated fitness went down.  fits/s = 1 / wall seconds to reach that level;
    when plain search does not reach it within the cap, the speed-up is a
    lower bound.  Reduced size (default): 256 replicates, 2^16 training
    trajectories, 1e5 screened and 1,000 re-simulated per generation; --full:
    512, 2^20, 1e6 and 10,000."""
    import torch
    from cutauleaping_b200 import fitsearch as fs
    full = a.full
    n_rep = 512 if full else 256
    n_traj = (1 << 20) if full else (1 << 16)
    screen = 1_000_000 if full else 100_000
    pop = 10_000 if full else 1000
    max_gen = 40 if full else 30
    p = fs.make_problem(n_rep=n_rep, samples=50, t_end=5.0)
    truth = float(fs.true_fitness(p, p.theta_true[None, :], seed=4242)[0])
    level = truth * 1.02

    def run_until(mode, offset, **kw):
        hist = fs.cem(p, mode=mode, generations=max_gen, pop=pop, seed=1, stop_at=level,
                      time_limit=a.time_limit, **kw)
        reached = hist[-1][2] <= level
        return offset + hist[-1][0], hist[-1][1], reached, hist
    torch.cuda.synchronize()
    plain_times, surr_times = [], []
    tp, sp, plain_ok, ph = run_until("plain", 0.0, times=plain_times)
    t0 = time.perf_counter()
    theta, traj = fs.training_data(p, n_traj)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net, sc = fs.train_surrogate(p, theta, traj, epochs=2, batch=16384)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0 - t_data
    ft_log = []
    ts, ss, surr_ok, sh = run_until("surrogate", t_data + t_train, screen=screen, keep_frac=0.01, net=net, sc=sc,
                                    inner=a.inner, finetune_steps=a.finetune, replay=(theta, traj), log=ft_log,
                                    times=surr_times)
    # the surrogate's own error where it matters: its predicted fitness at the
    # true parameters and at the best candidate found, against simulation
    pred = fs.predicted_fitness(p, net, sc, np.stack([p.theta_true, sh[-1][3]]))
    sim_best = float(fs.true_fitness(p, sh[-1][3][None, :], seed=4243)[0])
    scr = screen_roofline(p, net, sc, n_cand=200_000)
    print(json.dumps({
        "metric": METRIC, "config": {"workload": "surrogate-screened parameter estimation: 32x64 network "
                                                 "(generator seed 1), 8 unknown rate constants, target = mean "
                                                 f"of {n_rep} simulations at 50 instants", "full_size": full,
                                     "n_rep": n_rep, "training_trajectories": n_traj, "screened_per_gen": screen,
                                     "surrogate_iterations_per_gen": a.inner,
                                     "finetune_steps_per_gen": a.finetune,
                                     "resimulated_per_gen": pop, "max_generations": max_gen,
                                     "time_limit_s": a.time_limit},
        "roofline": scr, "gpu_launches": None,
        "value": 1.0 / ts, "unit": "fits/s (surrogate-screened)", "plain_fits_per_s": 1.0 / tp,
        "speedup_vs_plain": tp / ts, "speedup_is_lower_bound": not plain_ok, "surrogate_reached": surr_ok,
        "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
        "fitness": {"true_parameters": truth, "level": level, "plain_best": ph[-1][2], "surrogate_best": sh[-1][2]},
        "time_s": {"plain_to_level": tp, "surrogate_to_level": ts, "surrogate_data": t_data,
                   "surrogate_training": t_train},
        "generations": {"plain": len(ph), "surrogate": len(sh)},
        "per_generation_s": {
            "plain": [{k: round(v, 3) if isinstance(v, float) else v for k, v in x.items()} for x in plain_times],
            "surrogate": [{k: round(v, 3) if isinstance(v, float) else v for k, v in x.items()} for x in surr_times]},
        "surrogate_at": {"true_parameters": {"predicted": float(pred[0]), "simulated": truth},
                         "best_found": {"predicted": float(pred[1]), "simulated_again": sim_best}},
        "finetune": {"phases": len(ft_log), "kept": sum(1 for x in ft_log if x["kept"]),
                     "surrogate_error": [[round(x["surrogate_error_before"], 4), round(x["after"], 4)]
                                         for x in ft_log]},
        "simulations_to_level": {"plain": sp, "surrogate": ss},
        "curves": {"plain": [[round(h[0], 3), h[2]] for h in ph],
                   "surrogate": [[round(h[0] + t_data + t_train, 3), h[2]] for h in sh]},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--full", action="store_true", help="config 5 at the configured sizes")
    ap.add_argument("--inner", type=int, default=3,
                    help="config 5: surrogate-only CEM iterations per generation (3: 6.3x against 4.8x with 1 at "
                         "the reduced size, one B200)")
    ap.add_argument("--time-limit", type=float, default=None,
                    help="config 5: wall-second cap per search (a capped plain search makes the speed-up a lower bound)")
    ap.add_argument("--screen-only", action="store_true", help="config 5: time the fused screening kernel alone")
    ap.add_argument("--gemm-only", action="store_true", help="config 5: time the surrogate's training GEMM alone")
    ap.add_argument("--finetune", type=int, default=100,
                    help="config 5: surrogate fine-tuning steps per generation on the re-simulated trajectories")
    ap.add_argument("--sims", type=int, default=None, help="simulations per GPU (default: config's)")
    ap.add_argument("--group", type=int, default=0, help="lanes per simulation (0 = library choice)")
    ap.add_argument("--threads", type=int, default=0, help="threads per block (0 = library choice)")
    ap.add_argument("--min-blocks", type=int, default=0,
                    help="register budget of the sweep kernel: 2, 3 or 4 resident blocks (0 = library choice)")
    ap.add_argument("--sched", type=int, default=0,
                    help="scheduling: 1 block regrouping rounds, 2 warp-local (0 = library choice)")
    ap.add_argument("--flags", type=int, default=0, help="run flags (quirk switches; 1 = forced SSA)")
    ap.add_argument("--ssa-budget", type=int, default=0, help="SSA steps per simulation and round (0 = library)")
    ap.add_argument("--dec-budget", type=int, default=0, help="leap decisions per simulation and round (0 = library)")
    ap.add_argument("--warp-sims", type=int, default=0,
                    help="tiny networks: simulations per warp of the register-resident sweep "
                         "(0 = library choice, -1 = shared-memory sweep)")
    ap.add_argument("--autotune", action="store_true", help="measure launch shapes before timing")
    ap.add_argument("--no-autotune", action="store_true", help="config 3: library default shapes")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-io", action="store_true", help="skip timing the output files")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.config == 5 and a.gemm_only:
        if rank == 0 and a.impl == "ours":
            bench_gemm(a)
        return
    if a.config == 5 and a.screen_only:
        if rank == 0 and a.impl == "ours":
            bench_screen(a)
        return
    if a.config == 5:
        if rank == 0 and a.impl == "ours":
            bench_config5(a)
        elif rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "config 5 is a search benchmark; its "
                              "plain-simulator arm is reported inside the config-5 line"}), flush=True)
        return
    segs = workload(a.config, a.sims)
    desc = " + ".join(d for _, d in segs)
    n_total = sum(net.n for net, _ in segs)

    if a.impl == "reference":
        if rank != 0:
            return
        v, fv, meta = cpu_reference_segments(segs, a.steps, a.warmup, a.flags)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "sims/s",
            "firings_per_s": fv, "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": meta["sample_ms"], "ms_per_step_is": "one bounded sample step (see cpu_baseline.sample)",
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64/i32", "data": "synthetic",
            "config": {"workload": desc, "sims": n_total},
            "cpu_baseline": {"value": v, "unit": "sims/s", "cores": meta["cores"], "kind": "port",
                             "sample": meta["sample"]},
            "e2e": {"value": v, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
        return

    import torch
    import cutauleaping_b200 as ctl
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    parts = []
    for si, (net, _) in enumerate(segs):
        model = ctl.Model.create(net.left, net.right, net.feed, net.tvec, net.cs)
        n = net.n
        cfg = ctl.run_cfg(seed=1 + si, sim_base=rank * n, device=local, group=a.group, threads=a.threads,
                          min_blocks=a.min_blocks, sched=a.sched, flags=a.flags, ssa_budget=a.ssa_budget,
                          dec_budget=a.dec_budget, warp_sims=a.warp_sims,
                          uniform_rates=int(bool((net.c == net.c[0]).all())))
        X0 = torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).to(dev)
        c = torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).to(dev)
        out = torch.empty((n, model.ns, model.s_out), dtype=torch.int32, device=dev)
        info = torch.empty((n, 40), dtype=torch.uint8, device=dev)
        if a.autotune or (a.config == 3 and not a.no_autotune):
            # config 3 is defined with an autotuned block shape; the sample must
            # fill the GPU like the full batch does: a quarter of it, >= 16384
            model.autotune(n, X0.data_ptr(), c.data_ptr(), sample=min(n, max(16384, n // 4)), cfg=cfg)
        li = model.launch_info(n, cfg)
        graph = model.graph(n, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(),
                            stream.cuda_stream, cfg)
        parts.append(dict(net=net, model=model, cfg=cfg, X0=X0, c=c, out=out, info=info, li=li, graph=graph))
    # several segments (the uneven batch): one graph with a parallel branch per
    # segment, so that one segment's tail overlaps the other's work
    multi = None
    if len(parts) > 1:
        multi = ctl.graph_multi([(pt["model"], pt["net"].n, pt["X0"].data_ptr(), pt["c"].data_ptr(),
                                  pt["out"].data_ptr(), pt["info"].data_ptr(), pt["cfg"]) for pt in parts],
                                stream.cuda_stream)
    launchers = [multi] if multi is not None else [pt["graph"] for pt in parts]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    with torch.cuda.stream(stream):
        for _ in range(a.warmup):
            flush.fill_(1)
            for g in launchers:
                g.launch(stream.cuda_stream)
        stream.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(a.steps)]
        barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            for e0, e1 in ev:
                flush.fill_(1)
                e0.record(stream)
                for g in launchers:
                    g.launch(stream.cuda_stream)
                e1.record(stream)
            stream.synchronize()
        torch.cuda.synchronize()
        barrier()
    times = [e0.elapsed_time(e1) for e0, e1 in ev]
    ms = float(np.mean(times))
    if dist is not None:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    fire, ops, abytes = 0.0, 0.0, 0.0
    per_sim = {}
    for pt in parts:
        inf = pt["info"].cpu().numpy().view(ctl.INFO_DTYPE).reshape(-1)
        fire += float(inf["firings"].sum())
        ops += op_count(pt["net"], inf)
        abytes += algorithmic_bytes(pt["net"]) * pt["net"].n
        steps = inf["steps"].astype(np.float64)
        # step histogram: how simulations split between leap- and SSA-dominated regimes
        leap_share = inf["leaps"] / np.maximum(inf["leaps"] + inf["ssa_steps"], 1)
        per_sim[pt["net"].name] = {"steps": float(steps.mean()), "leaps": float(inf["leaps"].mean()),
                                   "ssa_steps": float(inf["ssa_steps"].mean()),
                                   "steps_quantiles": {q: float(np.percentile(steps, v)) for q, v in
                                                       (("p10", 10), ("p50", 50), ("p90", 90), ("p99", 99),
                                                        ("max", 100))},
                                   "leap_share_histogram": np.histogram(leap_share, bins=10,
                                                                        range=(0.0, 1.0))[0].tolist(),
                                   "status_ok": int((inf["status"] == 0).sum())}
    if dist is not None:
        f = torch.tensor([fire], dtype=torch.float64, device=dev)
        dist.all_reduce(f)
        fire = float(f.item())
    value = world * n_total / (ms * 1e-3)
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    li0 = parts[0]["li"]
    issue_peak = li0.sm_count * 128 * sm_mhz * 1e6  # FP32/INT32 lanes per SM x clock
    peaks, peak_src = measured_peaks()
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = None
    tf = os.path.join(ROOT, "profiles", "sweep_traffic.txt")
    if os.path.exists(tf) and a.config == 2 and n_total == 65536:
        try:
            line = open(tf).read().split("#")[0]
            traffic = float(line.split(":")[1]) / 1e9  # GB per launch
        except (OSError, ValueError, IndexError):
            traffic = None

    e2e = None
    if not a.no_e2e:
        import ctypes as C
        L = ctl.lib()
        host = []
        for pt in parts:
            net = pt["net"]
            host.append(dict(
                X0=torch.from_numpy(np.ascontiguousarray(net.X0, np.int32)).pin_memory(),
                c=torch.from_numpy(np.ascontiguousarray(net.c, np.float32)).pin_memory(),
                out=torch.empty((net.n, pt["model"].ns, pt["model"].s_out), dtype=torch.int32).pin_memory(),
                info=torch.empty((net.n, 40), dtype=torch.uint8).pin_memory()))

        def call_one(pt, h):
            st = L.ctl_run(pt["model"].handle, C.byref(pt["cfg"]), pt["net"].n, C.c_void_p(h["X0"].data_ptr()),
                           C.c_void_p(h["c"].data_ptr()), C.c_void_p(h["out"].data_ptr()),
                           C.c_void_p(h["info"].data_ptr()))
            if st not in (ctl.OK, ctl.ERR_STEP_LIMIT):
                raise ctl.CtlError(st, "ctl_run")

        def call():
            # one host thread per segment: the calls (each on its own streams)
            # run side by side, as the segments' branches do in the graph
            if len(parts) == 1:
                call_one(parts[0], host[0])
                return
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(len(parts)) as ex:
                list(ex.map(lambda ph: call_one(*ph), zip(parts, host)))
        call()
        barrier()
        et = []
        for _ in range(max(1, min(a.steps, 3))):
            t0 = time.perf_counter()
            call()
            et.append(time.perf_counter() - t0)
        e2e_s = float(np.mean(et))
        if dist is not None:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": world * n_total / e2e_s, "unit": "sims/s",
               "h2d_bytes_per_step": int(sum(h["X0"].numel() * 4 + h["c"].numel() * 4 for h in host)),
               "d2h_bytes_per_step": int(sum(h["out"].numel() * 4 + h["info"].numel() for h in host)),
               "ms_per_step": e2e_s * 1e3, "timer": "host perf_counter around ctl_run"}
        e2e["bit_identical_to_device_run"] = all(
            bool(np.array_equal(h["out"].numpy(), pt["out"].cpu().numpy())) for pt, h in zip(parts, host))

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        v, fv, meta = cpu_reference_segments(segs, 1, 0, a.flags)
        cpu = {"value": v, "unit": "sims/s", "cores": meta["cores"], "kind": "port",
               "sample": meta["sample"], "firings_per_s": fv}

    io = None
    if rank == 0 and not a.no_io:
        pt = parts[0]
        k = min(pt["net"].n, 4096)
        io = io_timing(pt["model"], pt["out"][:k].cpu().numpy().view(np.uint32))
        if "error" not in io:
            io["sample"] = f"the first {k} simulations' samples of {pt['net'].name}"

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "sims/s",
            "firings_per_s": fire / (ms * 1e-3),
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64/i32", "data": "synthetic",
            "config": {"workload": desc, "sims_per_gpu": n_total, "seed": 1,
                       "l2": "flushed between steps by a 256 MB device write",
                       "launch": [{"group": pt["li"].group, "threads": pt["li"].threads,
                                   "blocks": pt["li"].blocks, "slots_per_block": pt["li"].slots_per_block,
                                   "smem_bytes": pt["li"].smem_bytes, "regs": pt["li"].regs_per_thread,
                                   "min_blocks": pt["li"].min_blocks, "sched": pt["li"].sched,
                                   "ssa_budget": pt["li"].ssa_budget, "dec_budget": pt["li"].dec_budget,
                                   "warp_sims": pt["li"].warp_sims,
                                   "blocks_per_sm": pt["li"].blocks_per_sm} for pt in parts],
                       "autotuned": bool(a.autotune or (a.config == 3 and not a.no_autotune)),
                       "graph": ("one CUDA graph per step, a parallel branch per segment" if multi is not None
                                 else "one CUDA graph per step"),
                       "parallelism": f"dp{world} (independent simulations per rank)"},
            "roofline": {"bound": "hbm", "achieved": abytes / (ms * 1e-3) / 1e9,
                         "peak": hbm_peak, "unit": "GB/s",
                         "frac": abytes / (ms * 1e-3) / 1e9 / hbm_peak,
                         "traffic": traffic, "traffic_unit": "GB per launch (ncu, scaled)",
                         "algorithmic_gb_per_launch": abytes / 1e9,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peak_src == "measured"
                         else "fallback: 6,650 GB/s (earlier pool measurement)",
                         "note": "HBM is not the bound of this issue-bound kernel; see roofline_issue"},
            "roofline_issue": {"achieved": ops / (ms * 1e-3) / 1e12, "peak": issue_peak / 1e12,
                               "unit": "Tops/s", "frac": ops / (ms * 1e-3) / issue_peak,
                               "convention": "32-bit ops per SSA step / leap attempt (bench.op_count)",
                               "peak_source": f"{li0.sm_count} SMs x 128 FP32/INT32 lanes x median SM clock"},
            "gpu_launches": a.steps * len(parts),
            "clocks": clocks,
            "per_sim": per_sim,
        }
        if e2e is not None:
            line["e2e"] = e2e
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if io is not None:
            line["io"] = io
        print(json.dumps(line), flush=True)
    del launchers, multi
    for pt in parts:
        del pt["graph"]
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
