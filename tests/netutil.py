"""Shared helpers for the tests: small networks and oracle/GPU runners."""
import numpy as np

import oracle
from cutauleaping_b200 import inputs


def small_networks():
    """(name, Network) pairs covering orders 0-3, feed species, criticality."""
    nets = [("schlogl", inputs.schlogl(64, samples=40, t_end=2.0))]
    for S, R, seed, t_end, x0, sigma in [(4, 6, 3, 2.0, (5, 200), 0.0), (8, 12, 5, 2.0, (3, 300), 0.5),
                                         (16, 32, 7, 1.0, (10, 2000), 0.0),
                                         (32, 64, 11, 0.5, (10, 10000), 0.5)]:
        # sigma > 0: every simulation gets its own rate constants (per-row c path)
        net = inputs.synthetic(S, R, 48, seed=seed, t_end=t_end, samples=25, x0_range=x0,
                               perturb_sigma=sigma, perturb_seed=seed)
        nets.append((f"syn{S}x{R}" + ("p" if sigma else ""), net))
    # immigration-death with a feed species and an order-3 reaction
    left = np.array([[0, 0, 0], [1, 0, 0], [3, 0, 0], [1, 0, 1]], np.int32)
    right = np.array([[1, 0, 0], [0, 0, 0], [2, 1, 0], [0, 1, 1]], np.int32)
    n = 48
    X0 = np.tile(np.array([30, 0, 50], np.int32), (n, 1))
    c = np.tile(np.array([20.0, 0.5, 1e-3, 0.01]), (n, 1))
    nets.append(("feed3", inputs.Network(left, right, np.array([0, 0, 1], np.int32), X0, c,
                                         np.linspace(0.1, 3.0, 30), np.array([0, 1], np.int32))))
    return nets


def oracle_model(net, *, seed=0, flags=0, eps=0.03, nc=10, ssa_factor=10.0, ssa_steps=100,
                 max_steps=0xFFFFFFFF):
    return oracle.OracleModel(net.left, net.right, net.feed, net.tvec, net.cs, eps=eps, nc=nc,
                              ssa_factor=ssa_factor, ssa_steps=ssa_steps, flags=flags, seed=seed,
                              max_steps=max_steps)


def oracle_run(net, *, sim_base=0, **kw):
    m = oracle_model(net, **kw)
    return m.run(net.X0, np.asarray(net.c, np.float32), sim_base=sim_base)


def same_info(a, b):
    for f in ("t_final", "firings", "status", "steps", "leaps", "ssa_steps", "rejections"):
        if not np.array_equal(a[f], b[f]):
            return f
    return None
