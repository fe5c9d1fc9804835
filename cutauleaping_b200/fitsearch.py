"""Parameter estimation: plain-simulator search versus surrogate-screened search.

The reference's fitness mode (kernel.cu:365-423) scores candidate parameter
sets by simulating each of them p_rep times and comparing the ensemble mean
with a target time series (calculateFitness, 2phase_n-tau-leaping.cu:
3324-3408: sum over samples and species of |target - mean| / target, divided
by samples x species).  The optimiser that proposes candidates lives outside
the reference; here both searches use the same cross-entropy method (CEM) in
log-parameter space:

* plain:     every proposed candidate is simulated (n_rep simulations) and
             scored with the reference fitness;
* surrogate: every generation screens many candidates with the MLP
             surrogate (cutauleaping_b200.surrogate), re-simulates only the
             best 1% with the plain method and keeps the elite by that true
             fitness; the plain method is the fallback and the arbiter.

All simulation goes through the CUDA sweep (ctl_run_device) and the fitness
through calculateFitness on the device (ctl_fitness_device).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import CtlError, Model, OK, lib, run_cfg
from . import inputs
from . import shard
from . import surrogate as sg


@dataclass
class FitProblem:
    left: np.ndarray
    right: np.ndarray
    c_base: np.ndarray          # [R] rate constants (unknown ones replaced per candidate)
    X0: np.ndarray              # [S]
    tvec: np.ndarray            # [ns]
    unknown: np.ndarray         # [8] reaction indices
    theta_true: np.ndarray      # [8] log rate constants
    log_lo: np.ndarray
    log_hi: np.ndarray
    target: np.ndarray          # [ns][S] uint32 ensemble mean (rounded), the fitting target
    n_rep: int
    model: Model = field(repr=False, default=None)

    @property
    def S(self):
        return self.left.shape[1]


def make_problem(S=32, R=64, *, net_seed=1, theta_seed=2, n_rep=512, samples=50, t_end=5.0,
                 n_unknown=8, lo=1e-3, hi=1.0, sim_seed=77):
    """A config-2-style random network with `n_unknown` rate constants
    replaced by unknowns, their true values log-uniform in [lo, hi]; the
    target is the mean of n_rep simulations at the true values."""
    left, right, c, X0 = inputs.random_network(S, R, net_seed)
    rng = np.random.default_rng(theta_seed)
    order = left.sum(1)
    cand = np.flatnonzero(order >= 1)
    unknown = np.sort(rng.choice(cand, size=n_unknown, replace=False))
    theta_true = rng.uniform(math.log(lo), math.log(hi), size=n_unknown)
    tvec = t_end * np.arange(1, samples + 1) / samples
    p = FitProblem(left, right, c, X0, tvec, unknown, theta_true, np.full(n_unknown, math.log(lo)),
                   np.full(n_unknown, math.log(hi)), None, n_rep)
    p.model = Model.create(left, right, None, tvec)
    samples_ = simulate(p, theta_true[None, :], n_rep, seed=sim_seed, sim_base=1 << 30)
    mean = samples_.reshape(n_rep, samples, S).astype(np.float64).mean(0)
    p.target = np.rint(mean).astype(np.uint32)
    return p


def _rates(p: FitProblem, theta_log, n_rep, torch):
    n = theta_log.shape[0]
    c = torch.as_tensor(np.tile(p.c_base.astype(np.float32), (n, 1)), device="cuda")
    c[:, torch.as_tensor(p.unknown, device="cuda")] = torch.exp(
        torch.as_tensor(theta_log, dtype=torch.float32, device="cuda"))
    return c.repeat_interleave(n_rep, dim=0).contiguous()


def _sweep(p: FitProblem, theta_log, n_rep, seed, sim_base, torch):
    """Simulate n_rep copies of every candidate; returns device samples
    [n*n_rep][ns][S] (int32 view of the uint32 counts)."""
    n = theta_log.shape[0]
    N = n * n_rep
    c = _rates(p, theta_log, n_rep, torch)
    X0 = torch.as_tensor(np.tile(p.X0.astype(np.int32), (N, 1)), device="cuda")
    out = torch.empty((N, len(p.tvec), p.S), dtype=torch.int32, device="cuda")
    info = torch.empty((N, 40), dtype=torch.uint8, device="cuda")
    cfg = run_cfg(seed=seed, sim_base=sim_base, max_steps=20_000_000)
    p.model.run_device(N, X0.data_ptr(), c.data_ptr(), out.data_ptr(), info.data_ptr(),
                       torch.cuda.current_stream().cuda_stream, cfg)
    return out


def simulate(p: FitProblem, theta_log, n_rep, *, seed, sim_base=0):
    import torch
    return _sweep(p, np.asarray(theta_log), n_rep, seed, sim_base, torch).cpu().numpy().view(np.uint32)


def true_fitness(p: FitProblem, theta_log, *, seed, sim_base=0, chunk=256, keep_reps=0):
    """Reference fitness of each candidate from n_rep simulations, on the
    device.  With keep_reps > 0 also returns the first keep_reps trajectories
    of every candidate (device tensor [n*keep_reps][ns][S], candidate-major)."""
    import torch
    L = lib()
    theta_log = np.asarray(theta_log)
    n = theta_log.shape[0]
    tgt = torch.as_tensor(p.target.astype(np.uint32).view(np.int32).reshape(-1), device="cuda")
    fit = np.empty(n)
    kept = []
    for a in range(0, n, chunk):
        th = theta_log[a:a + chunk]
        k = th.shape[0]
        out = _sweep(p, th, p.n_rep, seed, sim_base + a * p.n_rep, torch)
        exp_id = torch.zeros(k, dtype=torch.uint8, device="cuda")
        f = torch.zeros(k * p.n_rep, dtype=torch.float64, device="cuda")
        st = L.ctl_fitness_device(C.c_void_p(out.data_ptr()), len(p.tvec), p.S, C.c_void_p(tgt.data_ptr()),
                                  C.c_void_p(exp_id.data_ptr()), 1, 1, 1, k * p.n_rep, p.n_rep,
                                  C.c_void_p(f.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        if st != OK:
            raise CtlError(st, "ctl_fitness_device")
        fit[a:a + k] = f[:k].cpu().numpy()
        if keep_reps:
            r = min(keep_reps, p.n_rep)
            kept.append(out.view(k, p.n_rep, len(p.tvec), p.S)[:, :r].reshape(k * r, len(p.tvec), p.S).clone())
    if keep_reps:
        return fit, torch.cat(kept)
    return fit


# ---------------------------------------------------------------------------
# Surrogate training data, training, screening
# ---------------------------------------------------------------------------

def training_data(p: FitProblem, n_traj, *, seed=5, sim_seed=91):
    """n_traj simulations, one per parameter set drawn from the prior box."""
    import torch
    rng = np.random.default_rng(seed)
    theta = rng.uniform(p.log_lo, p.log_hi, size=(n_traj, len(p.unknown)))
    out = _sweep(p, theta, 1, sim_seed, 1 << 31, torch)
    return torch.as_tensor(theta, dtype=torch.float32, device="cuda"), out


def train_surrogate(p: FitProblem, theta, traj, *, epochs=1, batch=16384, lr=2e-3, seed=0, log=None,
                    net=None, sc=None, steps=None, cosine=True, replay=None, dist=None):
    """Fit the MLP to (theta, t) -> counts of single trajectories (Gaussian
    NLL: the network learns the ensemble mean and log-variance).  With `net`
    and `sc` given, continues training that network (fine-tuning) with its
    output scaling unchanged; with `replay` = (theta0, traj0), half of every
    batch is drawn from that earlier data so the network keeps what it knew
    outside the new data's region.

    Data-parallel with `dist` (an initialised process group of several
    ranks, each holding its own shard of the trajectories): every rank
    draws its own batch, the gradients are averaged over ranks in one
    all-reduce before each Adam step (shard.allreduce_mean), and the output
    scaling is rank 0's, so all ranks keep identical weights."""
    import torch
    n, ns, S = traj.shape
    rank = dist.get_rank() if shard.multi_rank(dist) else 0
    if sc is None:
        # per-species scale from a sample of the trajectories
        ix = torch.randint(0, n, (min(n, 1 << 14),), device="cuda",
                           generator=torch.Generator(device="cuda").manual_seed(seed))
        ys = traj[ix].to(torch.float32)
        y_mean = ys.mean(dim=(0, 1))
        y_std = ys.std(dim=(0, 1)).clamp_min(1.0)
        shard.broadcast_([y_mean, y_std], dist)
        sc = sg.Scaling(p.log_lo, p.log_hi, float(p.tvec[-1]), y_mean.cpu().numpy(), y_std.cpu().numpy())
    else:
        y_mean = torch.as_tensor(sc.y_mean, dtype=torch.float32, device="cuda")
        y_std = torch.as_tensor(sc.y_std, dtype=torch.float32, device="cuda")
    tv = torch.as_tensor(p.tvec, dtype=torch.float32, device="cuda")
    if net is None:
        net = sg.MLP(S, seed=seed)
    total = n * ns
    steps = steps or max(1, (epochs * total) // batch)
    g = torch.Generator(device="cuda").manual_seed(seed + net.version + 7919 * rank)
    sources = [(theta, traj, batch if replay is None else batch // 2)]
    if replay is not None:
        sources.append((replay[0], replay[1], batch - batch // 2))
    hist = []
    for it in range(steps):
        Xs, Ts = [], []
        for th_, tr_, k in sources:
            idx = torch.randint(0, tr_.shape[0] * ns, (k,), device="cuda", generator=g)
            si, ti = idx // ns, idx % ns
            Xs.append(sg.make_inputs(th_[si], tv[ti], sc, torch))
            Ts.append((tr_[si, ti].to(torch.float32) - y_mean) / y_std)
        X = Xs[0] if len(Xs) == 1 else torch.cat(Xs)
        tgt = Ts[0] if len(Ts) == 1 else torch.cat(Ts)
        out = net.forward(X)
        loss, dW, db = net.backward(out, tgt)
        shard.allreduce_mean(dW + db, dist)
        rate = lr * 0.5 * (1 + math.cos(math.pi * it / steps)) if cosine else lr
        net.adam(dW, db, lr=rate)
        if log is not None and (it % 200 == 0 or it == steps - 1):
            hist.append((it, loss.item() / (batch * S)))
    if log is not None:
        log.extend(hist)
    net.check_error_flag()
    return net, sc


def predicted_fitness(p: FitProblem, net, sc, theta_log):
    """Reference fitness computed from the surrogate's ensemble mean, in the
    fused screening kernel (ctl_mlp_screen)."""
    import torch
    theta = torch.as_tensor(np.asarray(theta_log), dtype=torch.float32, device="cuda")
    return sg.screen(net, theta, p.tvec, p.target.astype(np.float32), sc).cpu().numpy()


def predicted_fitness_layers(p: FitProblem, net, sc, theta_log, *, chunk=65536):
    """The same fitness through the layer-by-layer path (one tcgen05 GEMM
    per layer, fitness in PyTorch): the cross-check of the fused kernel."""
    import torch
    theta_log = torch.as_tensor(np.asarray(theta_log), dtype=torch.float32, device="cuda")
    n = theta_log.shape[0]
    ns, S = len(p.tvec), p.S
    tv = torch.as_tensor(p.tvec, dtype=torch.float32, device="cuda")
    tgt = torch.as_tensor(p.target.astype(np.float64), device="cuda")
    ym = torch.as_tensor(sc.y_mean, device="cuda", dtype=torch.float64)
    ys = torch.as_tensor(sc.y_std, device="cuda", dtype=torch.float64)
    fit = torch.empty(n, dtype=torch.float64, device="cuda")
    per = max(1, chunk // ns)
    for a in range(0, n, per):
        th = theta_log[a:a + per]
        k = th.shape[0]
        rows = k * ns
        pad = (-rows) % 128
        X = sg.make_inputs(th.repeat_interleave(ns, 0), tv.repeat(k), sc, torch)
        if pad:
            X = torch.cat([X, torch.zeros(pad, X.shape[1], dtype=X.dtype, device="cuda")])
        y = net.forward(X, keep=False)[:rows, :S].to(torch.float64)
        mean = (y * ys + ym).view(k, ns, S)
        d = (tgt - mean).abs()
        d = torch.where(tgt != 0, d / tgt.clamp_min(1), d)
        fit[a:a + k] = d.sum(dim=(1, 2)) / (ns * S)
    return fit.cpu().numpy()


# ---------------------------------------------------------------------------
# Cross-entropy search
# ---------------------------------------------------------------------------

def _surrogate_error(p, net, sc, cand, f):
    """Mean relative error of the surrogate's fitness against simulated fitness."""
    pf = predicted_fitness(p, net, sc, cand)
    return float(np.mean(np.abs(pf - f) / np.maximum(f, 1e-12)))


def cem(p: FitProblem, *, mode, generations, pop, elite=0.1, screen=None, keep_frac=0.01, net=None,
        sc=None, seed=0, sim_seed=1000, time_limit=None, stop_at=None, inner=1, explore_frac=0.0,
        finetune_steps=0, finetune_reps=8, finetune_lr=2e-4, finetune_batch=8192, replay=None, log=None,
        times=None):
    """Cross-entropy search in log-parameter space.

    mode 'plain' simulates every one of `pop` candidates per generation.
    mode 'surrogate' runs, per generation, `inner` surrogate-only CEM
    iterations from the current proposal (each screens `screen` candidates
    and refits the proposal to the best `elite` fraction by predicted
    fitness; the last one keeps its screened set), then re-simulates the best
    max(pop, keep_frac * screen) screened candidates -- of which a fraction
    `explore_frac` is replaced by unscreened draws from the proposal -- and
    refits the proposal to their best by true fitness.

    With finetune_steps > 0 the surrogate is then fine-tuned on
    `finetune_reps` of the trajectories just simulated for half of those
    candidates (fresh optimiser moments, constant rate, half of every batch
    replayed from `replay` = the original training data when given), and the
    simulated fitness of the other half decides the outcome: the fine-tuned
    weights are kept only if the surrogate's error on that half went down.
    Every candidate whose fitness is reported was simulated.  Returns a list
    of (wall seconds, simulations so far, best true fitness, best theta), one
    entry per generation; `log`, if a list, receives per-generation notes, and
    `times`, if a list, each generation's seconds of screening, re-simulation
    (true fitness) and fine-tuning."""
    import torch
    rng = np.random.default_rng(seed)
    d = len(p.unknown)
    mu = (p.log_lo + p.log_hi) / 2
    sd = (p.log_hi - p.log_lo) / 2
    floor = 0.02 * (p.log_hi - p.log_lo)
    best_f, best_t = math.inf, None
    hist = []
    sims = 0
    t0 = time.perf_counter()
    for gen in range(generations):
        tg0 = time.perf_counter()
        t_screen = t_ft = 0.0
        if mode == "plain":
            cand = np.clip(rng.normal(mu, sd, size=(pop, d)), p.log_lo, p.log_hi)
        else:
            for it in range(inner):
                big = np.clip(rng.normal(mu, sd, size=(screen, d)), p.log_lo, p.log_hi)
                order = np.argsort(predicted_fitness(p, net, sc, big))
                if it < inner - 1:
                    el = big[order[: max(2, int(elite * keep_frac * screen))]]
                    mu = el.mean(0)
                    sd = np.maximum(el.std(0), floor)
            t_screen = time.perf_counter() - tg0
            nk = max(pop, int(keep_frac * screen))
            nx = int(explore_frac * nk)
            cand = big[order[: nk - nx]]
            if nx:
                cand = np.concatenate([cand, np.clip(rng.normal(mu, sd, size=(nx, d)), p.log_lo, p.log_hi)])
        tr0 = time.perf_counter()
        if mode != "plain" and finetune_steps:
            f, traj = true_fitness(p, cand, seed=sim_seed + gen, sim_base=0, keep_reps=finetune_reps)
        else:
            f = true_fitness(p, cand, seed=sim_seed + gen, sim_base=0)
        t_resim = time.perf_counter() - tr0
        sims += len(cand) * p.n_rep
        order = np.argsort(f)
        if f[order[0]] < best_f:
            best_f, best_t = float(f[order[0]]), cand[order[0]].copy()
        ne = max(2, int(elite * len(cand)))
        el = cand[order[:ne]]
        mu = el.mean(0)
        sd = np.maximum(el.std(0), floor)
        hist.append((time.perf_counter() - t0, sims, best_f, best_t))
        if times is not None:
            times.append({"gen": gen, "screen_s": t_screen, "resim_s": t_resim, "finetune_s": 0.0,
                          "candidates": int(len(cand)), "best": best_f})
        if time_limit is not None and time.perf_counter() - t0 > time_limit:
            break
        if stop_at is not None and best_f <= stop_at:
            break
        tf0 = time.perf_counter()
        if mode != "plain" and finetune_steps:
            reps = min(finetune_reps, p.n_rep)
            tr_idx, va_idx = np.arange(0, len(cand), 2), np.arange(1, len(cand), 2)
            before = _surrogate_error(p, net, sc, cand[va_idx], f[va_idx])
            saved = net.state()
            net.reset_optimizer()
            rows = torch.as_tensor((tr_idx[:, None] * reps + np.arange(reps)[None, :]).reshape(-1), device="cuda")
            th = torch.as_tensor(np.repeat(cand[tr_idx], reps, axis=0), dtype=torch.float32, device="cuda")
            train_surrogate(p, th, traj[rows], net=net, sc=sc, steps=finetune_steps, lr=finetune_lr,
                            batch=finetune_batch, cosine=False, replay=replay)
            after = _surrogate_error(p, net, sc, cand[va_idx], f[va_idx])
            kept = after < before
            if not kept:
                net.load_state(saved)
            if log is not None:
                log.append({"gen": gen, "surrogate_error_before": before, "after": after, "kept": bool(kept)})
        if times is not None:
            times[-1]["finetune_s"] = time.perf_counter() - tf0
    return hist
