"""Surrogate-screened parameter estimation on the GPU (reduced size).

A 32-species / 64-reaction network with 8 unknown rate constants; the target
is the ensemble mean of simulations at the true constants (config 5 of the
benchmark plan, scaled down so the test runs in about a minute).

* the surrogate is trained on trajectories the simulator produces and its
  predicted fitness ranks candidates: Spearman correlation with the true
  (re-simulated, calculateFitness) fitness > 0.5;
* what the trained network gains over the method without it: candidates it
  keeps from a proposal pool have a clearly lower true fitness than the same
  number taken without screening (equal simulation budget).
"""
import numpy as np
import pytest
from scipy.stats import spearmanr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from cutauleaping_b200 import fitsearch as fs
    p = fs.make_problem(n_rep=64, samples=25, t_end=2.0)
    theta, traj = fs.training_data(p, 1 << 15)
    log = []
    net, sc = fs.train_surrogate(p, theta, traj, epochs=2, batch=8192, log=log)
    return p, net, sc, log


def test_training_loss_decreases(trained):
    p, net, sc, log = trained
    assert log[-1][1] < log[0][1] - 0.5, log


def test_surrogate_ranks_candidates(trained):
    from cutauleaping_b200 import fitsearch as fs
    p, net, sc, _ = trained
    rng = np.random.default_rng(3)
    cand = rng.uniform(p.log_lo, p.log_hi, size=(256, len(p.unknown)))
    pf = fs.predicted_fitness(p, net, sc, cand)
    tf = fs.true_fitness(p, cand, seed=11)
    rho = spearmanr(pf, tf).correlation
    assert rho > 0.5, rho


def test_screening_gains_over_plain_sampling(trained):
    """What the trained network gains: from the same proposal distribution,
    the 64 candidates the surrogate keeps out of 6400 have a lower true
    (re-simulated) fitness than 64 candidates taken without it."""
    from cutauleaping_b200 import fitsearch as fs
    p, net, sc, _ = trained
    rng = np.random.default_rng(8)
    pool = rng.uniform(p.log_lo, p.log_hi, size=(6400, len(p.unknown)))
    kept = pool[np.argsort(fs.predicted_fitness(p, net, sc, pool))[:64]]
    plain = pool[:64]
    f_kept = fs.true_fitness(p, kept, seed=21)
    f_plain = fs.true_fitness(p, plain, seed=21)
    assert np.median(f_kept) < 0.8 * np.median(f_plain), (np.median(f_kept), np.median(f_plain))
    assert f_kept.min() <= f_plain.min()


@pytest.mark.parametrize("inner", [1, 3])
def test_search_runs_and_records_budget(trained, inner):
    from cutauleaping_b200 import fitsearch as fs
    p, net, sc, _ = trained
    plain = fs.cem(p, mode="plain", generations=2, pop=64, seed=1)
    surr = fs.cem(p, mode="surrogate", generations=2, pop=64, screen=6400, keep_frac=0.01, net=net, sc=sc, seed=1,
                  inner=inner)
    assert surr[-1][1] == plain[-1][1] == 2 * 64 * p.n_rep   # equal simulation budgets
    assert all(h[2] <= g[2] for g, h in zip(surr, surr[1:]))  # best fitness never worsens


def test_guarded_finetuning_keeps_or_restores(trained):
    """Fine-tuning on re-simulated trajectories is checked against simulated
    fitness on held-out candidates: the log says whether the new weights were
    kept, and a rejected phase leaves the surrogate's predictions unchanged."""
    from cutauleaping_b200 import fitsearch as fs
    p, net, sc, _ = trained
    theta, traj = fs.training_data(p, 1 << 12, seed=9)
    probe = np.random.default_rng(5).uniform(p.log_lo, p.log_hi, size=(64, len(p.unknown)))
    log = []
    before = net.state()
    fs.cem(p, mode="surrogate", generations=2, pop=64, screen=6400, keep_frac=0.01, net=net, sc=sc, seed=3,
           finetune_steps=20, replay=(theta, traj), log=log)
    assert len(log) == 2 and all(set(x) >= {"surrogate_error_before", "after", "kept"} for x in log)
    net.check_error_flag()
    pf_now = fs.predicted_fitness(p, net, sc, probe)
    assert np.isfinite(pf_now).all()
    if not any(x["kept"] for x in log):
        net2_pf = pf_now
        net.load_state(before)
        assert np.array_equal(fs.predicted_fitness(p, net, sc, probe), net2_pf)
    net.load_state(before)  # leave the module fixture as it was
