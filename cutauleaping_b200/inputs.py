"""Input folders in the reference's "BioSimWare" format, and seeded workloads.

Folder layout (read by 2phase_n-tau-leaping.cu:90-1261):
    left_side, right_side   R rows x S tab-separated stoichiometric coefficients
    M_feed                  one row of S flags (nonzero = species held constant)
    MX_0                    one row of S initial counts per simulation
    c_matrix                one row of R rate constants per simulation
    t_vector                sample instants, one per line (the last one is t_max)
    cs_vector               sampled species ids, one per line (optional)
    ts_rep, p_rep, ts_numtgt, tts_vector, ts_matrix   fitness targets (optional)

The generators stand in for inputs the reference does not ship (it has no
example folder): the Schlogl model of schlogl.xml and random mass-action
networks with the shapes and value distributions of the benchmark configs.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Network:
    left: np.ndarray            # [R][S] int32 reactant coefficients
    right: np.ndarray           # [R][S] int32 product coefficients
    feed: np.ndarray            # [S] int32, nonzero = held constant
    X0: np.ndarray              # [n][S] int32
    c: np.ndarray               # [n][R] float64
    tvec: np.ndarray            # [ns] float64
    cs: np.ndarray | None = None
    name: str = "network"
    meta: dict = field(default_factory=dict)

    @property
    def S(self):
        return self.left.shape[1]

    @property
    def R(self):
        return self.left.shape[0]

    @property
    def n(self):
        return self.X0.shape[0]

    def subset(self, idx) -> "Network":
        return Network(self.left, self.right, self.feed, self.X0[idx], self.c[idx], self.tvec,
                       self.cs, self.name, dict(self.meta))


def _fmt(x: float) -> str:
    return repr(float(x))


def write_folder(path: str, net: Network, target: dict | None = None) -> str:
    """Write `net` as an input folder the reference (and this CLI) can read."""
    os.makedirs(path, exist_ok=True)

    def rows(name, M, conv=str):
        with open(os.path.join(path, name), "w") as f:
            for r in np.atleast_2d(M):
                f.write("\t".join(conv(v) for v in r) + "\n")

    rows("left_side", net.left)
    rows("right_side", net.right)
    rows("M_feed", net.feed.reshape(1, -1))
    rows("MX_0", net.X0)
    rows("c_matrix", net.c, _fmt)
    with open(os.path.join(path, "t_vector"), "w") as f:
        f.write("".join(_fmt(t) + "\n" for t in net.tvec))
    if net.cs is not None:
        with open(os.path.join(path, "cs_vector"), "w") as f:
            f.write("".join(f"{int(s)}\n" for s in net.cs))
    if target is not None:
        for k in ("ts_rep", "p_rep", "ts_numtgt"):
            with open(os.path.join(path, k), "w") as f:
                f.write(f"{int(target[k])}\n")
        with open(os.path.join(path, "tts_vector"), "w") as f:
            f.write("".join(f"{int(v)}\n" for v in target["tts_vector"]))
        # ts_matrix: [ns][experiments][repetitions][species] -> one row per sample
        ts = np.asarray(target["ts_matrix"])
        with open(os.path.join(path, "ts_matrix"), "w") as f:
            for i in range(ts.shape[0]):
                f.write(_fmt(net.tvec[i]) + "\t" + "\t".join(str(int(v)) for v in ts[i].ravel()) + "\n")
    return path


def schlogl(n: int = 4096, *, samples: int = 100, t_end: float = 5.0) -> Network:
    """Schlogl bistable model (schlogl.xml): species A, X, B with A and B held
    constant (M_feed = 1 0 1); 2X+A->3X (3e-7), 3X->2X+A (1e-4), B->X (1e-3),
    X->B (3.5); A=1e5, X(0)=250, B=2e5; `samples` instants t_end*i/samples."""
    left = np.array([[1, 2, 0], [0, 3, 0], [0, 0, 1], [0, 1, 0]], np.int32)
    right = np.array([[0, 3, 0], [1, 2, 0], [0, 1, 0], [0, 0, 1]], np.int32)
    feed = np.array([1, 0, 1], np.int32)
    X0 = np.tile(np.array([100000, 250, 200000], np.int32), (n, 1))
    c = np.tile(np.array([3e-7, 1e-4, 1e-3, 3.5]), (n, 1))
    tvec = t_end * np.arange(1, samples + 1) / samples
    return Network(left, right, feed, X0, c, tvec, np.arange(3, dtype=np.int32), "schlogl")


def random_network(S: int, R: int, seed: int, *, c_range=(1e-4, 1.0), x0_range=(10, 10_000),
                   max_order=2):
    """Random mass-action network: per reaction the order (reactant molecules)
    is uniform in {0..max_order} and so is the product count, each molecule's
    species uniform over the S species (a species drawn twice gets
    stoichiometry 2); reactions with no net change are redrawn.  Rate
    constants log-uniform in c_range, initial counts log-uniform integers in
    x0_range.  Returns (left, right, c[R], X0[S])."""
    rng = np.random.default_rng(seed)
    left = np.zeros((R, S), np.int32)
    right = np.zeros((R, S), np.int32)
    r = 0
    while r < R:
        lo = rng.integers(0, max_order + 1)
        po = rng.integers(0, max_order + 1)
        L = np.zeros(S, np.int32)
        Pr = np.zeros(S, np.int32)
        for s in rng.integers(0, S, size=lo):
            L[s] += 1
        for s in rng.integers(0, S, size=po):
            Pr[s] += 1
        if np.array_equal(L, Pr):
            continue
        left[r], right[r] = L, Pr
        r += 1
    c = np.exp(rng.uniform(np.log(c_range[0]), np.log(c_range[1]), size=R))
    X0 = np.floor(np.exp(rng.uniform(np.log(x0_range[0]), np.log(x0_range[1] + 1), size=S)))
    X0 = np.clip(X0, x0_range[0], x0_range[1]).astype(np.int32)
    return left, right, c, X0


def synthetic(S: int, R: int, n: int, *, seed: int, t_end: float, samples: int,
              c_range=(1e-4, 1.0), x0_range=(10, 10_000), perturb_sigma: float = 0.0,
              perturb_seed: int = 0) -> Network:
    """A random network (random_network) replicated over n simulations; with
    perturb_sigma > 0 every simulation gets c * exp(sigma * z), z ~ N(0, 1)."""
    left, right, c, X0 = random_network(S, R, seed, c_range=c_range, x0_range=x0_range)
    Cm = np.tile(c, (n, 1))
    if perturb_sigma > 0:
        z = np.random.default_rng(perturb_seed).standard_normal((n, R))
        Cm = Cm * np.exp(perturb_sigma * z)
    tvec = t_end * np.arange(1, samples + 1) / samples
    return Network(left, right, np.zeros(S, np.int32), np.tile(X0, (n, 1)), Cm, tvec, None,
                   f"synthetic{S}x{R}", {"seed": seed})
