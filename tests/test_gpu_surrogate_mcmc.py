"""What the trained surrogate gains: delayed-acceptance MCMC against plain
engine MCMC on the 256-phase problem, on the GPU.

* the device sub-chain (lcb_surrogate_subchain) makes the same moves as the
  host loop that calls the surrogate once per move, on the same random numbers;
* the surrogate is trained on light curves the engine generates and its error
  is measured against the engine on held-out parameters;
* from one burned-in ensemble, delayed acceptance mixes faster per light
  curve the engine computes and per second than plain MCMC.  Mixing is the
  mean squared jump of the walkers in units of the plain chain's spread,
  which is robust on chains too short for autocorrelation times.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    return (importlib.import_module("lcurve-rs_b200.surrogate"), importlib.import_module("lcurve-rs_b200.mcmc"),
            importlib.import_module("lcurve-rs_b200.workloads"))


def _msjd(run, sig):
    d = np.diff(run.chain, axis=0) / sig
    return float(np.mean(np.sum(d * d, axis=2)))


def _problem(S, W):
    setup = S.CurveSetup()
    fid = S.CurveEngine(setup).curves(S.TRUTH[None, :])[0]
    data = W.noisy_data(setup.times, fid, setup.expose, setup.ndiv, seed=42)
    return setup, data


@pytest.mark.parametrize("move", ["stretch", "kde"])
def test_device_subchain_matches_host_loop(lcb, mods, move):
    S, M, W = mods
    setup, data = _problem(S, W)
    sur = S.Surrogate(seed=2)  # untrained weights are enough to compare the two paths
    sur.bind_data(data)
    rng = np.random.default_rng(0)
    walkers = M.initial_walkers(128, S.TRUTH, seed=1, spread=0.05)
    y, comp = walkers[:64], walkers[64:]
    ls = -0.5 * sur.chisq(y)
    rnd = M.subchain_numbers(rng, 6, 64, move)
    yd, lsd = sur.subchain(y, ls, comp, rnd, move=move)
    yh, lsh = M.subchain_host(sur, y, ls, comp, rnd, move=move)
    same = np.all(np.isclose(yd, yh, rtol=1e-12, atol=0), axis=1)
    # identical moves except where float rounding of the network input decides a tie
    assert same.mean() >= 0.95
    assert np.allclose(lsd[same], lsh[same], rtol=1e-6, atol=1e-6)
    assert np.any(np.any(yd != y, axis=1))


def test_trained_surrogate_gains_over_plain_mcmc(lcb, mods):
    S, M, W = mods
    setup, data = _problem(S, W)
    n, hold = 393216, 2048
    theta = S.sample_prior(n + hold, seed=11)
    curves = S.generate_curves(setup, theta)
    assert np.isfinite(curves).all()
    sur = S.Surrogate(seed=1)
    losses = sur.fit(theta[:n], curves[:n], epochs=250)
    assert losses[-1] < 0.01 * losses[0]
    rel = S.scaled_rel_error(sur.predict(theta[n:]), curves[n:])
    assert np.median(rel) < 1.5e-3, np.median(rel)  # surrogate vs the engine it stands in for

    eng = S.CurveEngine(setup, data=data)
    sur.bind_data(data)
    start = M.run_delayed(eng, sur, M.initial_walkers(256, S.TRUTH, seed=3), 300, seed=4, substeps=32).chain[-1]
    # one-time costs outside the timed runs: a resident batch (and its captured graph) for every
    # engine batch size, and the sub-chain graph of this move
    for size in eng.sizes:
        eng.chisq(start[:size])
    M.run_plain(eng, start, 3, seed=6, move="kde", bandwidth=0.6)
    M.run_delayed(eng, sur, start, 3, seed=6, substeps=2, move="kde", bandwidth=0.6)
    # same move (KDE proposals from the other half) with and without the surrogate screen, 256 walkers
    plain = M.run_plain(eng, start, 200, seed=5, move="kde", bandwidth=0.6)
    da = M.run_delayed(eng, sur, start, 200, seed=5, substeps=2, move="kde", bandwidth=0.6)
    sig = plain.chain.reshape(-1, 5).std(axis=0)
    per_eval = (_msjd(da, sig) / da.engine_evals) / (_msjd(plain, sig) / plain.engine_evals)
    per_s = (_msjd(da, sig) / da.seconds) / (_msjd(plain, sig) / plain.seconds)
    print(f"jump distance gain of delayed acceptance: per engine evaluation {per_eval:.2f}, per second {per_s:.2f}")
    # per evaluation the gain is fixed by the seeds (4.7 measured); per second it is wall clock of
    # 200-step runs on a shared host (1.7 measured), hence the looser bound; the benchmark reports
    # the ESS/s ratio of long chains
    assert per_eval > 3.0 and per_s > 1.3, (per_eval, per_s, da.acceptance, plain.acceptance)


def test_sharded_samplers_over_nccl_match_one_process(mods):
    """The samplers' rank sharding through an NCCL group (device tensors in the
    all-gather) of one rank: the chains of the unsharded run, exactly."""
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    S, M, _ = mods

    class Quadratic:  # a cheap stand-in likelihood: only the sharding is under test here
        evals = 0

        def chisq(self, th, scale=True):
            th = np.atleast_2d(th)
            self.evals += th.shape[0]
            return np.sum(((th - S.TRUTH) / (0.02 * (S.PRIOR_HI - S.PRIOR_LO))) ** 2, axis=1)

    p0 = M.initial_walkers(32, S.TRUTH, seed=1, spread=0.02)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        a = M.run_plain(Quadratic(), p0, 30, seed=2, move="kde", group=dist.group.WORLD)
    finally:
        dist.destroy_process_group()
    b = M.run_plain(Quadratic(), p0, 30, seed=2, move="kde")
    assert np.array_equal(a.chain, b.chain) and a.engine_evals == b.engine_evals
