"""The CPU oracle against exact answers and against the reference binary.

1. Exact answers: immigration-death and pure decay have closed-form laws;
   forced SSA (LightweightSSA semantics) must reproduce them, and the Schlogl
   model must match the independent FP64 Gillespie direct method.
2. The reference itself: tests/golden/reference_*.npz hold statistics of
   trajectories printed by the reference binary built from its own sources
   (tests/golden/make_reference_fixtures.py).  The oracle, run on the same
   inputs with its own random stream, must agree within 3 standard errors
   (family-wise bounds in tests/stats.py) and pass Bonferroni-corrected
   two-sample KS tests.
"""
import glob
import math
import os
import sys

import numpy as np
import pytest
from scipy.stats import binom, poisson

import oracle
from cutauleaping_b200 import inputs
from tests import stats
from tests.netutil import oracle_model

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _net(left, right, x0, c, tvec, n, feed=None):
    left = np.array(left, np.int32)
    right = np.array(right, np.int32)
    S = left.shape[1]
    return inputs.Network(left, right, np.zeros(S, np.int32) if feed is None else np.array(feed, np.int32),
                          np.tile(np.array(x0, np.int32), (n, 1)), np.tile(np.array(c, float), (n, 1)),
                          np.asarray(tvec, float), None)


def _run(net, flags=0, seed=3, mode=0):
    m = oracle_model(net, seed=seed, flags=flags)
    return m.run(net.X0, net.c.astype(np.float32), mode=mode)[0]


def test_immigration_death_ssa_is_exact():
    # 0 -> X (k), X -> 0 (mu), X(0) = 0: X(t) ~ Poisson(k/mu (1 - e^{-mu t}))
    k, mu, n = 40.0, 0.8, 6000
    tv = np.array([0.25, 0.5, 1.0, 2.0, 4.0])
    out = _run(_net([[0], [1]], [[1], [0]], [0], [k, mu], tv, n), flags=oracle.FORCE_SSA)[:, :, 0]
    for i, t in enumerate(tv):
        lam = k / mu * (1 - math.exp(-mu * t))
        x = out[:, i].astype(float)
        assert abs(x.mean() - lam) < 4 * math.sqrt(lam / n)
        hist = np.bincount(out[:, i], minlength=int(lam * 3) + 20)
        support = np.arange(len(hist))
        expct = poisson.pmf(support, lam) * n
        keep = expct > 5
        chi2 = float((((hist[keep] - expct[keep]) ** 2) / expct[keep]).sum())
        assert chi2 < keep.sum() + 5 * math.sqrt(2 * keep.sum())


def test_pure_decay_ssa_is_binomial():
    N0, mu, n = 400, 0.5, 6000
    tv = np.array([0.3, 1.0, 2.5])
    out = _run(_net([[1]], [[0]], [N0], [mu], tv, n), flags=oracle.FORCE_SSA)[:, :, 0]
    for i, t in enumerate(tv):
        p = math.exp(-mu * t)
        x = out[:, i].astype(float)
        assert abs(x.mean() - N0 * p) < 4 * math.sqrt(N0 * p * (1 - p) / n)
        assert abs(x.var() / (N0 * p * (1 - p)) - 1) < 4 * math.sqrt(2 / n)
        # whole distribution: Kolmogorov distance to Binomial(N0, p) within
        # the 1 % critical value (conservative for a discrete law)
        k = np.arange(N0 + 1)
        emp = np.searchsorted(np.sort(x), k, side="right") / n
        assert np.max(np.abs(emp - binom.cdf(k, N0, p))) < 1.63 / math.sqrt(n)


def test_immigration_death_tau_leaping_mean():
    # Leap-dominated regime (X ~ 1e4).  For a linear network the leap mean
    # follows the explicit Euler recursion m' = m (1 - mu tau) + k tau, which
    # overshoots the exact mean by O(eps) (about 1% at eps = 0.03, t = 2).
    k, mu, n = 2.0e4, 1.0, 2000
    tv = np.array([0.5, 1.0, 2.0])
    out = _run(_net([[0], [1]], [[1], [0]], [0], [k, mu], tv, n))[:, :, 0].astype(float)
    for i, t in enumerate(tv):
        lam = k / mu * (1 - math.exp(-mu * t))
        assert 0.0 < out[:, i].mean() / lam - 1 < 0.02


@pytest.mark.parametrize("flags", [0, oracle.FORCE_SSA])
def test_schlogl_matches_exact_gillespie(flags):
    net = inputs.schlogl(6000, samples=40, t_end=4.0)
    m = oracle_model(net, seed=11, flags=flags)
    ours, _ = m.run(net.X0, net.c.astype(np.float32))
    exact, _ = m.gillespie(net.X0, net.c.astype(np.float32))
    a, b = ours[:, :, 1].astype(float), exact[:, :, 1].astype(float)
    n = a.shape[0]
    ok, info = stats.check_means(a.mean(0), a.var(0, ddof=1), n, b.mean(0), b.var(0, ddof=1), n)
    assert ok, info
    ps = stats.ks_pvalues(a[:, 4::5], b[:, 4::5])
    assert ps.min() > 0.01 / len(ps), ps


def test_dimerisation_matches_exact_gillespie():
    # 2X -> 0 with inflow: order-2 propensity 0.5 X (X-1)
    net = _net([[0], [2]], [[1], [0]], [300], [200.0, 0.01], np.linspace(0.2, 3, 15), 5000)
    m = oracle_model(net, seed=5)
    ours, _ = m.run(net.X0, net.c.astype(np.float32))
    exact, _ = m.gillespie(net.X0, net.c.astype(np.float32))
    a, b = ours[:, :, 0].astype(float), exact[:, :, 0].astype(float)
    ok, info = stats.check_means(a.mean(0), a.var(0, ddof=1), len(a), b.mean(0), b.var(0, ddof=1), len(b))
    assert ok, info


# ---------------------------------------------------------------------------
# The reference binary's own trajectories
# ---------------------------------------------------------------------------

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "reference_*.npz")))


def _cases():
    sys.path.insert(0, GOLDEN)
    import make_reference_fixtures as mk
    return mk.CASES


@pytest.mark.skipif(not FIXTURES, reason="no reference fixtures in tests/golden")
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[10:-4] for p in FIXTURES])
def test_oracle_matches_reference_binary(path):
    name = os.path.basename(path)[len("reference_"):-len(".npz")]
    factory, threads, blocks, force, keep = _cases()[name]
    g = np.load(path)
    net = factory()
    m = oracle_model(net, seed=2024, flags=oracle.FORCE_SSA if force else 0)
    ours, _ = m.run(net.X0, net.c.astype(np.float32))
    x = ours.astype(np.float64)
    n = x.shape[0]
    assert int(g["n"]) == n
    ok, info = stats.check_means(x.mean(0), x.var(0, ddof=1), n, g["mean"], g["var"], n)
    assert ok, f"{name}: {info}"
    raw_idx, raw = g["raw_idx"], g["raw"]
    ours_raw = ours[:, raw_idx][:, :, list(g["raw_species"])]
    ps = stats.ks_pvalues(ours_raw, raw)
    assert ps.min() > 0.01 / len(ps), f"{name}: KS p-values {np.sort(ps)[:5]}"
    vz = [stats.var_z(ours_raw[:, i, j], raw[:, i, j]) for i in range(raw.shape[1]) for j in range(raw.shape[2])]
    vz = np.abs(np.array(vz))
    assert vz.max() < 4.5 and (vz > 3).mean() <= 0.05, f"{name}: variance z {np.sort(vz)[-5:]}"


@pytest.mark.parametrize("S,R,seed,t_end,samples,extra", [
    (64, 128, 0, 10.0, 200, {}),                                                   # config 2
    (32, 64, 3, 10.0, 200, {}),                                                    # config 3, synthetic part
    (512, 1024, 0, 20.0, 500, {"c_range": (1e-5, 1e-1), "x0_range": (1, 100000)}),  # config 4
])
def test_benchmark_networks_pass_the_pilot_rule(S, R, seed, t_end, samples, extra):
    """The benchmark's synthetic networks keep the generator's acceptance
    rule: in a 64-simulation pilot no recorded count reaches 2^30 (far from
    the int32 limit, so no run can end in OVERFLOW) and every simulation
    finishes normally."""
    from cutauleaping_b200 import inputs
    from tests.netutil import oracle_run
    net = inputs.synthetic(S, R, 64, seed=seed, t_end=t_end, samples=samples, **extra)
    out, info = oracle_run(net, seed=1)
    assert int(out.max()) < 2 ** 30
    assert (info["status"] == 0).all()
