"""The samplers' logic on the CPU, with a Gaussian stand-in for the engine.

Delayed acceptance must leave the engine's posterior unchanged whatever the
surrogate: here the surrogate is deliberately wrong (shifted mean, wrong
widths), and the delayed-acceptance chains must still reproduce the target's
mean and spread, as the plain chains do.  Tolerances: 0.15 sigma on means and
15% on standard deviations (Monte Carlo error of ~60k correlated samples).
"""
import importlib

import numpy as np
import pytest


@pytest.fixture(scope="module")
def M():
    return importlib.import_module("lcurve-rs_b200.mcmc")


@pytest.fixture(scope="module")
def S():
    return importlib.import_module("lcurve-rs_b200.surrogate")


class Gaussian:
    """chisq of a Gaussian in the parameters (widths 2% of the prior box)."""

    def __init__(self, S, mu, frac, shift=0.0):
        self.mu = mu + shift * frac * (S.PRIOR_HI - S.PRIOR_LO)
        self.sig = frac * (S.PRIOR_HI - S.PRIOR_LO)
        self.evals = 0

    def chisq(self, theta, scale=True):
        theta = np.atleast_2d(theta)
        self.evals += theta.shape[0]
        return np.sum(((theta - self.mu) / self.sig) ** 2, axis=1)


def _check(run, target, burn=0.3):
    ch = run.chain[int(burn * run.chain.shape[0]):].reshape(-1, run.chain.shape[2])
    assert np.all(np.abs(ch.mean(0) - target.mu) < 0.15 * target.sig), (ch.mean(0), target.mu)
    assert np.all(np.abs(ch.std(0) / target.sig - 1.0) < 0.15), ch.std(0) / target.sig


def test_plain_and_delayed_sample_the_engine_posterior(M, S):
    mu = 0.5 * (S.PRIOR_LO + S.PRIOR_HI)
    eng = Gaussian(S, mu, 0.02)
    bad = Gaussian(S, mu, 0.03, shift=0.7)  # wrong centre and widths
    p0 = M.initial_walkers(64, mu, seed=1, spread=0.02)
    plain = M.run_plain(eng, p0, 1500, seed=2)
    _check(plain, eng)
    for k in (1, 4):
        eng.evals = 0
        da = M.run_delayed(eng, bad, p0, 1500, seed=3 + k, substeps=k)
        _check(da, eng)
        assert da.engine_evals == eng.evals <= 64 + 1500 * 64


def test_kde_moves_sample_the_engine_posterior(M, S):
    mu = 0.5 * (S.PRIOR_LO + S.PRIOR_HI)
    eng = Gaussian(S, mu, 0.02)
    bad = Gaussian(S, mu, 0.03, shift=0.7)
    p0 = M.initial_walkers(64, mu, seed=1, spread=0.02)
    _check(M.run_plain(eng, p0, 600, seed=2, move="kde"), eng)
    _check(M.run_delayed(eng, bad, p0, 600, seed=3, substeps=4, move="kde"), eng)


def test_kde_density_and_draws(M):
    rng = np.random.default_rng(0)
    comp = rng.normal(size=(200, 5)) * np.array([1.0, 2.0, 0.5, 3.0, 1.0])
    kde = M.KDE.of(comp)
    r = M.subchain_numbers(rng, 1, 20000, "kde", 5)[0]
    y = kde.draw(r)
    # the KDE's covariance is S (1 + h^2): draws spread slightly wider than the walkers
    h2 = 200 ** (-2.0 / 9)
    assert np.allclose(y.std(0), comp.std(0, ddof=1) * np.sqrt(1 + h2), rtol=0.05)
    # logq is the log of the mixture density up to one constant
    lq = kde.logq(y[:5])
    diff = y[:5, None, :] - comp[None]
    dens = np.exp(-0.5 * np.einsum("nmi,ij,nmj->nm", diff, kde.prec, diff)).sum(1)
    assert np.allclose(lq, np.log(dens))


def test_delayed_acceptance_with_the_exact_surrogate_accepts_every_screened_move(M, S):
    mu = 0.5 * (S.PRIOR_LO + S.PRIOR_HI)
    eng = Gaussian(S, mu, 0.02)
    p0 = M.initial_walkers(32, mu, seed=1, spread=0.02)
    da = M.run_delayed(eng, Gaussian(S, mu, 0.02), p0, 50, seed=9, substeps=3)
    assert da.accepted == da.stage1_pass > 0


def test_integrated_time_of_an_ar1_chain(M):
    rng = np.random.default_rng(0)
    n, w, rho = 20000, 8, 0.9
    x = np.zeros((n, w, 1))
    for t in range(1, n):
        x[t] = rho * x[t - 1] + rng.standard_normal((w, 1))
    tau = M.integrated_time(x)[0]
    assert abs(tau - (1 + rho) / (1 - rho)) < 0.1 * (1 + rho) / (1 - rho)


def _sharded_worker(rank, world, port, out):
    import os
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        out[rank] = _sharded_runs(dist.group.WORLD)
    finally:
        dist.destroy_process_group()


def _sharded_runs(group):
    M = importlib.import_module("lcurve-rs_b200.mcmc")
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    mu = 0.5 * (S.PRIOR_LO + S.PRIOR_HI)
    eng = Gaussian(S, mu, 0.02)
    p0 = M.initial_walkers(34, mu, seed=1, spread=0.02)  # halves of 17: uneven shards
    plain = M.run_plain(eng, p0, 40, seed=2, move="kde", group=group)
    da = M.run_delayed(eng, Gaussian(S, mu, 0.03, shift=0.7), p0, 40, seed=3, substeps=2, group=group)
    return plain.chain, da.chain, plain.engine_evals, da.engine_evals


def test_sharded_engine_evaluations_give_the_single_process_chains():
    """Two gloo ranks, each evaluating its share of every batch of proposals:
    both hold exactly the chains of one process, with the evaluations split."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.Manager().dict()
    mp.spawn(_sharded_worker, args=(2, port, out), nprocs=2, join=True)
    single = _sharded_runs(None)
    for r in (0, 1):
        assert np.array_equal(out[r][0], single[0]) and np.array_equal(out[r][1], single[1])
    assert out[0][2] + out[1][2] == single[2] and out[0][3] + out[1][3] == single[3]
    assert 0 < out[0][2] < single[2]


@pytest.mark.parametrize("sampler", ["plain", "delayed"])
def test_checkpoint_resume_reproduces_the_uninterrupted_chain(M, S, tmp_path, sampler):
    """A run stopped after its checkpoint and resumed from it gives the
    uninterrupted run's chain bit for bit (same positions, counters)."""
    mu = 0.5 * (S.PRIOR_LO + S.PRIOR_HI)
    p0 = M.initial_walkers(32, mu, seed=1, spread=0.02)

    def run(nsteps, ck=None):
        eng = Gaussian(S, mu, 0.02)
        if sampler == "plain":
            return M.run_plain(eng, p0, nsteps, seed=9, move="kde", checkpoint=ck)
        return M.run_delayed(eng, Gaussian(S, mu, 0.03, shift=0.5), p0, nsteps, seed=9, substeps=3, move="kde",
                             checkpoint=ck)

    full = run(60)
    ck = M.Checkpoint(tmp_path / "chain.npz", every=25)
    run(25, ck)   # "interrupted" after its checkpoint at step 25
    assert ck.path.exists()
    resumed = run(60, M.Checkpoint(ck.path, every=0))
    assert np.array_equal(resumed.chain, full.chain)
    assert (resumed.accepted, resumed.proposals, resumed.engine_evals) == \
           (full.accepted, full.proposals, full.engine_evals)
    assert resumed.stage1_pass == full.stage1_pass and resumed.surrogate_evals == full.surrogate_evals
