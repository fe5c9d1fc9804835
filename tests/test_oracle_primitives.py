"""Oracle primitives against known answers (CPU only).

Philox4x32-10 against the Random123 known-answer vectors of Salmon et al.
(SC'11); the own log/exp/log-factorial against libm; the Poisson sampler
against the exact Poisson pmf (chi-square over quantile bins, plus mean and
variance within 4 standard errors).
"""
import math

import numpy as np
import pytest
from scipy.stats import chisquare, poisson

import oracle


@pytest.mark.parametrize("ctr,key,expect", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox_known_answers(ctr, key, expect):
    assert list(oracle.philox(ctr, key)) == expect


def _ulps(a, b):
    return abs(a - b) / math.ulp(b)


def test_log_within_two_ulp():
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-740, 709, 5000)), rng.uniform(0.5, 2.0, 5000),
                         [1.0, 2.0, 0.5, 1e-310, 5e-324, 1.7976931348623157e308]])
    worst = max(_ulps(oracle.log(x), math.log(x)) for x in xs)
    assert worst <= 2.0
    assert oracle.log(1.0) == 0.0


def test_exp_within_one_ulp():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(-700, 0, 5000), rng.uniform(-12, 0, 5000), [0.0, -1e-300]])
    worst = max(_ulps(oracle.exp(x), math.exp(x)) for x in xs)
    assert worst <= 1.0
    assert oracle.exp(0.0) == 1.0


def test_logfact():
    for k in list(range(0, 40)) + [100, 1000, 12345, 10**6, 10**9]:
        assert abs(oracle.logfact(k) - math.lgamma(k + 1)) <= 2e-15 * max(1.0, math.lgamma(k + 1))


@pytest.mark.parametrize("lam", [0.01, 0.7, 3.0, 9.999, 10.0, 31.4, 250.0, 4.0e4, 2.5e6])
def test_poisson_distribution(lam):
    n = 30000
    ks = np.array([oracle.poisson(lam, 11, s, 2, 0, s % 7) for s in range(n)], dtype=np.int64)
    se = math.sqrt(lam / n)
    assert abs(ks.mean() - lam) < 4 * se
    # relative standard error of a Poisson sample variance: sqrt((1/lam + 2) / n)
    assert abs(ks.var() / lam - 1) < 4 * math.sqrt((1 / lam + 2) / n)
    qs = np.unique(poisson.ppf(np.linspace(0.002, 0.998, 30), lam).astype(np.int64))
    edges = np.concatenate([[-1], qs, [np.iinfo(np.int64).max // 2]])
    obs = np.histogram(ks, bins=edges + 0.5)[0]
    expct = (poisson.cdf(edges[1:], lam) - poisson.cdf(edges[:-1], lam)) * n
    keep = expct > 5
    p = chisquare(obs[keep], expct[keep] * obs[keep].sum() / expct[keep].sum()).pvalue
    assert p > 1e-3


def test_poisson_zero_rate_and_stream_independence():
    assert oracle.poisson(0.0, 1, 2, 3, 4, 5) == 0
    a = [oracle.poisson(50.0, 1, 0, 0, 0, r) for r in range(64)]
    b = [oracle.poisson(50.0, 1, 0, 0, 1, r) for r in range(64)]
    assert a != b  # different rejection attempt -> different stream
    assert a == [oracle.poisson(50.0, 1, 0, 0, 0, r) for r in range(64)]  # counter-based: repeatable
