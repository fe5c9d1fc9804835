"""The drop-in command line on the GPU, end to end.

`cutauleaping input threads blocks gpu offset out prefix fitness force_ssa
verbose` (kernel.cu:74-436) must write the per-simulation files of
WriteDynamics2 (2phase_n-tau-leaping.cu:3431-3469) with the oracle's samples,
honour `offset` (rows and random streams of a larger run), force SSA, print
dynamics to stdout with verbose = 2, write one binary sample file with
CTL_BINARY_OUTPUT=1, write a JSON run report with CTL_REPORT, and print calculateFitness
(3324-3408) values in fitness mode 2 -- checked against a numpy restatement.
"""
import os
import subprocess

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs
from tests.netutil import oracle_model

pytestmark = pytest.mark.gpu


def _rows(tvec, samples):
    return "".join("%g" % t + "".join(f"\t{v}" for v in samples[i]) + "\n" for i, t in enumerate(tvec))


def _cli(args, env_extra=None, cwd=None):
    env = dict(os.environ, CTL_SEED="5", **(env_extra or {}))
    return subprocess.run([ctl.CLI_PATH, *map(str, args)], capture_output=True, text=True, env=env, cwd=cwd,
                          timeout=300)


@pytest.fixture(scope="module")
def folder(tmp_path_factory):
    net = inputs.schlogl(48, samples=30, t_end=1.5)
    return inputs.write_folder(str(tmp_path_factory.mktemp("cli") / "schlogl"), net), net


@pytest.mark.parametrize("force", [0, 1])
def test_cli_files_match_oracle(folder, tmp_path, force):
    path, net = folder
    p = _cli([path, 8, 4, 0, 8, tmp_path / "out", "pref", 0, force, 0])
    assert p.returncode == 0, p.stderr
    ref, _ = oracle_model(net, seed=5, flags=force).run(net.X0[8:40], net.c[8:40].astype(np.float32), sim_base=8)
    for gid in range(32):
        got = open(tmp_path / "out" / f"pref_{gid}").read()
        assert got == _rows(net.tvec, ref[gid]), f"simulation {gid}"


def test_cli_binary_output_matches_oracle(folder, tmp_path):
    """CTL_BINARY_OUTPUT=1: one <prefix>.ctlbin with the same samples the
    text files carry, and no per-simulation files."""
    path, net = folder
    p = _cli([path, 8, 2, 0, 8, tmp_path / "ob", "pref", 0, 0, 0], {"CTL_BINARY_OUTPUT": "1"})
    assert p.returncode == 0, p.stderr
    ref, _ = oracle_model(net, seed=5).run(net.X0[8:24], net.c[8:24].astype(np.float32), sim_base=8)
    d = ctl.read_samples_binary(str(tmp_path / "ob" / "pref.ctlbin"))
    assert np.array_equal(np.asarray(d["samples"]), ref)
    assert np.array_equal(d["t"], np.asarray(net.tvec, np.float64))
    assert sorted(os.listdir(tmp_path / "ob")) == ["pref.ctlbin"]


def test_cli_run_report(folder, tmp_path):
    """CTL_REPORT=<path>: a JSON run report whose sums match the oracle's
    per-simulation records."""
    import json
    path, net = folder
    rep = tmp_path / "report.json"
    p = _cli([path, 8, 2, 0, 8, tmp_path / "or", "pref", 0, 0, 0], {"CTL_REPORT": str(rep)})
    assert p.returncode == 0, p.stderr
    _, info = oracle_model(net, seed=5).run(net.X0[8:24], net.c[8:24].astype(np.float32), sim_base=8)
    r = json.loads(rep.read_text())
    assert r["simulations"] == 16 and r["status"]["ok"] == 16 and r["seconds"] > 0
    assert r["firings"] == int(info["firings"].sum()) and r["steps"] == int(info["steps"].sum())
    assert r["launch"]["group"] >= 1 and r["launch"]["threads"] >= 32


def test_cli_stdout_dynamics(folder, tmp_path):
    path, net = folder
    p = _cli([path, 4, 2, 0, 0, tmp_path / "o2", "p", 0, 0, 2])
    assert p.returncode == 0, p.stderr
    ref, _ = oracle_model(net, seed=5).run(net.X0[:8], net.c[:8].astype(np.float32))
    exp = "".join(_rows(net.tvec, ref[g]) + "\n" for g in range(8))
    assert p.stdout.endswith(exp)


def _calc_fitness(samples, target, swarm, threads, p_rep):
    """calculateFitness (tau.cu:3324-3408) restated in numpy, same rounding."""
    N, ns, so = samples.shape
    nsets = N // p_rep
    out = np.zeros(N)
    for tid in range(nsets):
        b, t = divmod(tid, threads)
        ex = swarm[tid]
        sub = np.float32(0.0)
        for c in range(ns):
            for s in range(so):
                acc = 0.0
                for par in range(p_rep):
                    acc += float(samples[(b * p_rep + par) * threads + t, c, s])
                acc /= p_rep
                for e in range(target.shape[2]):
                    tgt = int(target[c, ex, e, s])
                    dist = abs(float(tgt) - acc)
                    if tgt != 0:
                        dist /= tgt
                    sub = np.float32(np.float64(sub) + dist)
        out[tid] = (1.0 / ns) * (1.0 / so) * float(sub)
    return out


def test_cli_fitness_stdout(tmp_path):
    net = inputs.schlogl(16, samples=8, t_end=0.4)
    rng = np.random.default_rng(1)
    ts = rng.integers(0, 400, size=(8, 2, 2, 3))
    target = {"ts_rep": 2, "p_rep": 2, "ts_numtgt": 3, "tts_vector": [8, 16], "ts_matrix": ts}
    path = inputs.write_folder(str(tmp_path / "fit"), net, target)
    p = _cli([path, 4, 4, 0, 0, tmp_path / "o", "pref", 2, 0, 0])
    assert p.returncode == 0, p.stderr
    samples, _ = oracle_model(net, seed=5).run(net.X0, net.c.astype(np.float32))
    swarm = np.array([0] * 8 + [1] * 8)
    fit = _calc_fitness(samples, ts, swarm, 4, 2)
    exp = "".join("".join("%g\t" % fit[sw * 4 + part] for part in range(4)) + "\t" for sw in range(4 // 2))
    assert p.stdout == "\n" * 2 + exp
