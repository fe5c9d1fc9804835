"""Generate statistical golden fixtures from the reference binary itself.

The reference (aresio/cuTauLeaping) ships no tests, golden outputs or example
inputs, and seeds cuRAND from time(NULL) (kernel.cu:176), so its output can
only be pinned statistically.  This script runs the reference binary built
from its own sources (oracle/_ref/cuTauLeaping, see oracle/Makefile) on
seeded input folders written by cutauleaping_b200.inputs, parses the dynamics
it prints (PrintDynamics2, 2phase_n-tau-leaping.cu:3472-3507, selected with
verbose = 2) and stores per-sample means and variances plus the raw values at
a few sample instants, so that tests can compare the CPU oracle against the
reference's own trajectories (3-standard-error and two-sample KS checks).

Run on a machine with a GPU (the reference has no CPU path):
    python tests/golden/make_reference_fixtures.py --out tests/golden

With --time it instead times the reference binary on the Schlogl benchmark
workload (4,096 simulations, t_end 5, 100 samples, 64 threads x 64 blocks):
the reference's own timer around its simulation loop (" * RUNNING TIME",
kernel.cu:240-347, printed with verbose = 1; file output comes after it),
three runs, printed as one JSON line.
"""
import json
import argparse
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cutauleaping_b200 import inputs  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "cuTauLeaping")

def _syn12x20():
    """12 species / 20 reactions (generator seed 0), with reaction 0 replaced
    by a zero-order inflow ->X0 at rate 1.  The reference's critical-reaction
    search (2phase_n-tau-leaping.cu:1993-2006) starts from PROP[0] and can walk
    past the last reaction when PROP[0] == 0 and the FP32-rounded target
    exceeds the critical sum; a positive zero-order reaction 0 keeps every
    read of that loop in bounds."""
    net = inputs.synthetic(12, 20, 4096, seed=0, t_end=2.0, samples=50, x0_range=(20, 2000))
    net.left[0] = 0
    net.right[0] = 0
    net.right[0, 0] = 1
    net.c[:, 0] = 1.0
    return net


def _syn32x64p():
    """The uneven batch's synthetic segment: 32 species / 64 reactions
    (generator seed 3), t_end 10, 200 samples, every simulation with its own
    rate constants c * exp(0.5 z) (perturbation seed 31), 30 threads x 137
    blocks = 4,110 simulations (the reference's shared memory holds 30
    simulations of this network per block).  Reaction 0 is replaced by the
    same positive zero-order inflow as in _syn12x20 (rate 1 in every row), so
    the reference's critical-reaction search stays in bounds."""
    net = inputs.synthetic(32, 64, 30 * 137, seed=3, t_end=10.0, samples=200, perturb_sigma=0.5,
                           perturb_seed=31)
    net.left[0] = 0
    net.right[0] = 0
    net.right[0, 0] = 1
    net.c[:, 0] = 1.0
    return net


# name -> (network factory, threads, blocks, force_ssa, species columns kept raw)
CASES = {
    "schlogl": (lambda: inputs.schlogl(4096), 64, 64, False, [1]),
    "schlogl_ssa": (lambda: inputs.schlogl(4096), 64, 64, True, [1]),
    "syn12x20": (_syn12x20, 32, 128, False, list(range(12))),
    "syn32x64p": (_syn32x64p, 30, 137, False, list(range(0, 32, 4))),
}
RAW_EVERY = 10  # keep raw values at every 10th sample instant


def parse_print_dynamics(text: str, n: int, ns: int, so: int) -> np.ndarray:
    """Rows `t<TAB>x...` per simulation, a blank line after each (PrintDynamics2)."""
    out = np.zeros((n, ns, so), dtype=np.uint32)
    sim, row = 0, 0
    for line in text.splitlines():
        if not line.strip():
            if row:
                if row != ns:
                    raise ValueError(f"simulation {sim}: {row} rows, expected {ns}")
                sim, row = sim + 1, 0
            continue
        if line.startswith(" *") or line.startswith("T=") or line.startswith("WARNING"):
            continue
        parts = line.split("\t")
        if len(parts) != so + 1:
            continue
        out[sim, row] = [int(v) for v in parts[1:]]
        row += 1
    if sim != n:
        raise ValueError(f"parsed {sim} simulations, expected {n}")
    return out


def run_case(name, factory, threads, blocks, force, keep, outdir):
    net = factory()
    n = threads * blocks
    assert net.n == n
    with tempfile.TemporaryDirectory() as td:
        folder = inputs.write_folder(os.path.join(td, name), net)
        args = [REF_BIN, folder, str(threads), str(blocks), "0", "0", os.path.join(td, "out"),
                "pref", "0", "1" if force else "0", "2"]
        t0 = time.time()
        p = subprocess.run(args, capture_output=True, text=True, timeout=1200)
        wall = time.time() - t0
        if p.returncode != 0:
            raise RuntimeError(f"{name}: reference exited {p.returncode}: {p.stderr[-2000:]}")
    so = net.S if net.cs is None else len(net.cs)
    samples = parse_print_dynamics(p.stdout, n, len(net.tvec), so)
    x = samples.astype(np.float64)
    raw_idx = np.arange(RAW_EVERY - 1, len(net.tvec), RAW_EVERY)
    path = os.path.join(outdir, f"reference_{name}.npz")
    np.savez_compressed(
        path, mean=x.mean(axis=0), var=x.var(axis=0, ddof=1), n=n, tvec=net.tvec,
        raw_idx=raw_idx, raw=samples[:, raw_idx][:, :, keep].astype(np.uint32), raw_species=keep,
        force_ssa=force, wall_s=wall, threads=threads, blocks=blocks)
    print(f"{name}: {n} simulations, reference wall {wall:.2f}s -> {path}", flush=True)


def time_reference(runs=3):
    """Seconds of the reference's own simulation-loop timer on the Schlogl
    benchmark workload, per run."""
    net = inputs.schlogl(4096)
    times = []
    with tempfile.TemporaryDirectory() as td:
        folder = inputs.write_folder(os.path.join(td, "schlogl"), net)
        for i in range(runs):
            out = os.path.join(td, f"out{i}")
            args = [REF_BIN, folder, "64", "64", "0", "0", out, "pref", "0", "0", "1"]
            p = subprocess.run(args, capture_output=True, text=True, timeout=900)
            if p.returncode != 0:
                raise RuntimeError(f"reference exited {p.returncode}: {p.stderr[-2000:]}")
            t = [float(l.split(":")[1].split()[0]) for l in p.stdout.splitlines() if "RUNNING TIME" in l]
            if not t:
                raise RuntimeError("no RUNNING TIME line in the reference's output")
            times.append(t[-1])
    return times


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--time", action="store_true", help="time the reference binary on the Schlogl workload")
    a = ap.parse_args()
    if not os.path.exists(REF_BIN):
        sys.exit(f"{REF_BIN} missing: build it with `make -C oracle ref` where the reference sources exist")
    if a.time:
        t = time_reference()
        print(json.dumps({"workload": "Schlogl, 4096 simulations, t_end 5, 100 samples, 64 threads x 64 blocks",
                          "reference_running_time_s": t, "sims_per_s_best": 4096 / min(t)}), flush=True)
        return
    os.makedirs(a.out, exist_ok=True)
    for name in a.cases:
        run_case(name, *CASES[name], a.out)


if __name__ == "__main__":
    main()
