"""Affine-invariant ensemble MCMC over the light-curve likelihood, plain and
with surrogate delayed acceptance.

The plain sampler is the reference fitter's emcee run
(python/lcurve_rs/fitting.py:536-600): walkers move by the stretch move
(Goodman & Weare 2010, a = 2) in two halves, each half's proposals evaluated
as one batch; log probability = log prior (uniform box) - chisq / 2 with
chisq from the light-curve engine (chisq_batch with scale=True,
fitting.py:329-341).

The delayed-acceptance sampler (Christen & Fox 2005) screens moves with
the surrogate first.  Each half-step, every walker of the moving half runs
`substeps` stretch moves against the (fixed) other half under the surrogate
posterior alone,

  stage 1  each sub-step accepted with min(1, z^(d-1) exp(l~(y) - l~(x)))
           l~ = surrogate log probability,

which is a kernel reversible with respect to the surrogate posterior; only a
walker whose sub-chain moved it from x to y is then decided by the engine,

  stage 2  accept y with min(1, exp(l(y) - l(x) - l~(y) + l~(x)))
           l = engine log probability,

else it stays at x.  Moves are the stretch move or, as emcee's KDEMove, an
independence proposal from a Gaussian KDE of the other half (valid because
that half is held fixed); the plain sampler offers the same two moves.
With substeps = 1 this is Christen & Fox's two-stage
delayed acceptance; with more sub-steps it is the surrogate transition method
(Liu 2001, sec. 9.4.3).  Either way the pair of stages satisfies detailed
balance with respect to the engine's posterior, so both samplers target the
same distribution and the engine decides every accepted move.

Multi-GPU: given a torch.distributed process group (one rank per GPU, every
rank with the same seed, start and surrogate), both samplers shard the
engine's work: every rank draws the same proposals, evaluates its contiguous
share of the rows that need the engine, and an all-gather returns every
row's log probability to every rank, so all ranks take the same decisions and
hold the same chain as one process would.  `engine_evals` counts the rank's
own evaluations.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from .surrogate import PARAMS, PRIOR_HI, PRIOR_LO


def log_prior(theta: np.ndarray) -> np.ndarray:
    theta = np.atleast_2d(theta)
    inside = np.all((theta >= PRIOR_LO) & (theta <= PRIOR_HI), axis=1)
    return np.where(inside, 0.0, -np.inf)


def _loglike(chisq: np.ndarray) -> np.ndarray:
    ll = -0.5 * np.asarray(chisq, dtype=np.float64)
    ll[~np.isfinite(ll)] = -np.inf
    return ll


def _stretch(rng, xs, xc, a):
    """Stretch proposals for the walkers xs against the complementary half xc."""
    n, d = xs.shape
    z = ((a - 1.0) * rng.random(n) + 1.0) ** 2 / a
    j = rng.integers(0, xc.shape[0], n)
    return xc[j] + z[:, None] * (xs - xc[j]), z


@dataclasses.dataclass
class KDE:
    """Gaussian KDE of the complementary walkers (emcee's KDEMove): kernel
    covariance h^2 S with S their sample covariance and h Scott's factor
    m^(-1/(d+4)).  Proposals from it are independent of the moving walker,
    which is what keeps the move valid with the complement held fixed."""

    comp: np.ndarray
    chol: np.ndarray   # kernel covariance = chol chol^T
    prec: np.ndarray   # its inverse
    white: np.ndarray  # chol^-1: whitened differences white (y - c) have |.|^2 = (y-c)^T prec (y-c)

    @classmethod
    def of(cls, comp: np.ndarray, bandwidth: float = 1.0) -> "KDE":
        """bandwidth multiplies Scott's factor (1 = emcee's default)."""
        m, d = comp.shape
        h2 = (bandwidth * m ** (-1.0 / (d + 4))) ** 2
        c = comp - comp.mean(axis=0)
        cov = (c.T @ c) * (h2 / (m - 1))  # the sample covariance (np.cov's), scaled
        cov[np.diag_indices(d)] += 1e-12 * np.diag(cov) + 1e-300
        chol = np.linalg.cholesky(cov)
        white = np.linalg.inv(chol)
        return cls(comp, chol, white.T @ white, white)

    def logq(self, y: np.ndarray) -> np.ndarray:
        # squared Mahalanobis distances |a - b|^2 = |a|^2 + |b|^2 - 2 a.b of whitened points, centred
        # on the components' mean so the coordinates are O(1) and the expansion loses nothing
        c0 = self.comp.mean(axis=0)
        yw = (np.atleast_2d(y) - c0) @ self.white.T
        cw = (self.comp - c0) @ self.white.T
        d2 = np.einsum("ni,ni->n", yw, yw)[:, None] + np.einsum("mi,mi->m", cw, cw)[None, :] - 2.0 * (yw @ cw.T)
        e = -0.5 * np.maximum(d2, 0.0)
        mx = e.max(axis=1, keepdims=True)
        return mx[:, 0] + np.log(np.exp(e - mx).sum(axis=1))

    def draw(self, r: np.ndarray) -> np.ndarray:
        """Proposals for one move: r[:, 0] picks the component, r[:, 3:] are normals."""
        m = self.comp.shape[0]
        j = np.minimum((r[:, 0] * m).astype(np.int64), m - 1)
        return self.comp[j] + r[:, 3:] @ self.chol.T


MOVES = ("stretch", "kde")


def subchain_numbers(rng, steps: int, n: int, move: str = "stretch", d: int = 5) -> np.ndarray:
    """steps x n x R random numbers of a surrogate sub-chain: a uniform for the
    stretch factor (or the KDE component), a uniform for the partner, ln of a
    uniform for acceptance, and for the KDE move d standard normals."""
    r = rng.random((steps, n, 3))
    with np.errstate(divide="ignore"):
        r[..., 2] = np.log(r[..., 2])
    if move == "kde":
        r = np.concatenate([r, rng.standard_normal((steps, n, d))], axis=2)
    return r


def subchain_host(surrogate, y, ls, comp, rnd, a=2.0, move="stretch", bandwidth=1.0):
    """The surrogate sub-chain on the host, one surrogate call per move; the
    same arithmetic as the device sub-chain (lcb_surrogate_subchain)."""
    y, ls = y.copy(), ls.copy()
    n, d = y.shape
    m = comp.shape[0]
    kde = KDE.of(comp, bandwidth) if move == "kde" else None
    lq = kde.logq(y) if kde else None
    for r in rnd:
        if kde:
            yp = kde.draw(r)
            lqp = kde.logq(yp)
            lratio = lq - lqp
        else:
            z = ((a - 1.0) * r[:, 0] + 1.0) ** 2 / a
            j = np.minimum((r[:, 1] * m).astype(np.int64), m - 1)
            yp = comp[j] + z[:, None] * (y - comp[j])
            lratio = (d - 1) * np.log(z)
        prior = log_prior(yp)
        lsp = prior + _loglike(surrogate.chisq(yp, scale=True))
        take = np.isfinite(prior) & (r[:, 2] < lratio + lsp - ls)
        y[take] = yp[take]
        ls[take] = lsp[take]
        if kde:
            lq[take] = lqp[take]
    return y, ls


@dataclasses.dataclass
class Run:
    chain: np.ndarray            # (nsteps, nwalkers, ndim)
    seconds: float               # wall time of the sampling loop
    engine_evals: int            # light curves computed by the engine
    surrogate_evals: int = 0
    stage1_pass: int = 0
    proposals: int = 0
    accepted: int = 0

    @property
    def acceptance(self) -> float:
        return self.accepted / max(self.proposals, 1)


class Checkpoint:
    """Sampler state saved every `every` steps to `path` (.npz: positions, log
    probabilities, the chain so far, counters, elapsed seconds and the random
    generator's state), from which a run resumes exactly: the resumed chain is
    the uninterrupted one, step for step and bit for bit.  The reference's
    fitter keeps its emcee chains in memory only (python/lcurve_rs/
    fitting.py:590-601)."""

    def __init__(self, path, every: int):
        import pathlib  # noqa: PLC0415
        self.path = pathlib.Path(path)
        self.every = int(every)

    def due(self, step: int) -> bool:
        return self.every > 0 and (step + 1) % self.every == 0

    def save(self, rng, step: int, chain: np.ndarray, seconds: float, **arrays) -> None:
        import json  # noqa: PLC0415
        tmp = self.path.with_name(self.path.name + ".tmp.npz")
        np.savez(tmp, step=step, chain=chain[:step], seconds=seconds,
                 rng=np.array(json.dumps(rng.bit_generator.state)), **arrays)
        tmp.replace(self.path)

    def load(self):
        """(step, chain prefix, seconds, rng state, other arrays) or None."""
        import json  # noqa: PLC0415
        if not self.path.exists():
            return None
        with np.load(self.path) as z:
            other = {k: z[k] for k in z.files if k not in ("step", "chain", "seconds", "rng")}
            return int(z["step"]), z["chain"], float(z["seconds"]), json.loads(str(z["rng"])), other


def shard_bounds(n: int, world: int) -> list[int]:
    """Row r of n belongs to rank k when bounds[k] <= r < bounds[k + 1]."""
    return [k * n // world for k in range(world + 1)]


def _gather_rows(local: np.ndarray, n: int, group) -> np.ndarray:
    """All ranks' contiguous shards (shard_bounds) of n float64 values, in rank order."""
    import torch  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415
    world = dist.get_world_size(group)
    b = shard_bounds(n, world)
    width = max(b[k + 1] - b[k] for k in range(world))
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.zeros(max(width, 1), dtype=torch.float64, device=dev)
    buf[:local.shape[0]] = torch.as_tensor(local, dtype=torch.float64)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return np.concatenate([parts[k][:b[k + 1] - b[k]].cpu().numpy() for k in range(world)])


def _eval_engine(engine, theta, chunk=128, group=None):
    if group is not None:  # this rank's share, then every rank's values
        import torch.distributed as dist  # noqa: PLC0415
        b = shard_bounds(theta.shape[0], dist.get_world_size(group))
        r = dist.get_rank(group)
        return _gather_rows(_eval_engine(engine, theta[b[r]:b[r + 1]], chunk), theta.shape[0], group)
    out = np.full(theta.shape[0], -np.inf)
    for i in range(0, theta.shape[0], chunk):
        out[i:i + chunk] = _loglike(engine.chisq(theta[i:i + chunk], scale=True))
    return out


def _eval_prob(engine, theta, group=None):
    lp = log_prior(theta)
    ok = np.isfinite(lp)
    out = np.full(theta.shape[0], -np.inf)
    if ok.any():
        out[ok] = lp[ok] + _eval_engine(engine, theta[ok], group=group)
    return out


def run_plain(engine, p0: np.ndarray, nsteps: int, seed: int = 0, a: float = 2.0, move: str = "stretch",
              bandwidth: float = 1.0, group=None, checkpoint: Checkpoint | None = None) -> Run:
    """The plain sampler; with `checkpoint`, its state is saved every
    checkpoint.every steps and a run whose checkpoint file exists resumes
    from it."""
    rng = np.random.default_rng(seed)
    x = np.array(p0, dtype=np.float64)
    nw, d = x.shape
    half = nw // 2
    chain = np.empty((nsteps, nw, d))
    t0 = time.perf_counter()
    ev0 = engine.evals
    acc = props = first = 0
    state = checkpoint.load() if checkpoint else None
    if state is not None:
        first, prefix, done_s, rng.bit_generator.state, o = state
        chain[:first] = prefix
        x, lp = o["x"].copy(), o["lp"].copy()
        acc, props = int(o["counts"][0]), int(o["counts"][1])
        ev0 -= int(o["counts"][2])
        t0 -= done_s
    else:
        lp = _eval_prob(engine, x, group)
    for s in range(first, nsteps):
        perm = rng.permutation(nw)
        for h in (0, 1):
            S, Cc = (perm[:half], perm[half:]) if h == 0 else (perm[half:], perm[:half])
            if move == "kde":
                kde = KDE.of(x[Cc], bandwidth)
                y = kde.draw(subchain_numbers(rng, 1, len(S), "kde", d)[0])
                lratio = kde.logq(x[S]) - kde.logq(y)
            else:
                y, z = _stretch(rng, x[S], x[Cc], a)
                lratio = (d - 1) * np.log(z)
            lpy = _eval_prob(engine, y, group)
            loga = lratio + lpy - lp[S]
            take = np.log(rng.random(len(S))) < loga
            x[S[take]] = y[take]
            lp[S[take]] = lpy[take]
            acc += int(take.sum())
            props += len(S)
        chain[s] = x
        if checkpoint and checkpoint.due(s):
            checkpoint.save(rng, s + 1, chain, time.perf_counter() - t0, x=x, lp=lp,
                            counts=np.array([acc, props, engine.evals - ev0]))
    return Run(chain, time.perf_counter() - t0, engine.evals - ev0, proposals=props, accepted=acc)


def run_delayed(engine, surrogate, p0: np.ndarray, nsteps: int, seed: int = 0, a: float = 2.0,
                substeps: int = 1, device_subchain: bool | None = None, move: str = "stretch",
                bandwidth: float = 1.0, group=None, checkpoint: Checkpoint | None = None) -> Run:
    """The delayed-acceptance sampler; `checkpoint` as in run_plain."""
    rng = np.random.default_rng(seed)
    x = np.array(p0, dtype=np.float64)
    nw, d = x.shape
    half = nw // 2
    chain = np.empty((nsteps, nw, d))
    t0 = time.perf_counter()
    ev0 = engine.evals
    on_device = hasattr(surrogate, "subchain") if device_subchain is None else device_subchain
    acc = props = passed = nsur = first = 0
    state = checkpoint.load() if checkpoint else None
    if state is not None:
        first, prefix, done_s, rng.bit_generator.state, o = state
        chain[:first] = prefix
        x, lp, lps = o["x"].copy(), o["lp"].copy(), o["lps"].copy()
        acc, props, passed, nsur = (int(v) for v in o["counts"][:4])
        ev0 -= int(o["counts"][4])
        t0 -= done_s
    else:
        lp = _eval_prob(engine, x, group)
        lps = log_prior(x) + _loglike(surrogate.chisq(x, scale=True))
    for s in range(first, nsteps):
        perm = rng.permutation(nw)
        for h in (0, 1):
            S, Cc = (perm[:half], perm[half:]) if h == 0 else (perm[half:], perm[:half])
            # stage 1: a surrogate sub-chain for every walker of the half
            rnd = subchain_numbers(rng, substeps, len(S), move, d)
            if on_device:
                y, lsy = surrogate.subchain(x[S], lps[S], x[Cc], rnd, a, move=move, bandwidth=bandwidth)
            else:
                y, lsy = subchain_host(surrogate, x[S], lps[S], x[Cc], rnd, a, move=move, bandwidth=bandwidth)
            nsur += substeps * len(S)
            moved = np.any(y != x[S], axis=1)
            # stage 2: the engine decides for the walkers that moved
            if moved.any():
                idx = np.nonzero(moved)[0]
                lpy = log_prior(y[idx]) + _eval_engine(engine, y[idx], group=group)
                loga2 = lpy - lp[S[idx]] - (lsy[idx] - lps[S[idx]])
                take = np.log(rng.random(len(idx))) < loga2
                w = S[idx[take]]
                x[w] = y[idx[take]]
                lp[w] = lpy[take]
                lps[w] = lsy[idx[take]]
                acc += int(take.sum())
                passed += len(idx)
            props += len(S)
        chain[s] = x
        if checkpoint and checkpoint.due(s):
            checkpoint.save(rng, s + 1, chain, time.perf_counter() - t0, x=x, lp=lp, lps=lps,
                            counts=np.array([acc, props, passed, nsur, engine.evals - ev0]))
    return Run(chain, time.perf_counter() - t0, engine.evals - ev0, surrogate_evals=nsur, stage1_pass=passed,
               proposals=props, accepted=acc)


# ---------------------------------------------------------------------------
# effective sample size (integrated autocorrelation time, emcee's estimator)
# ---------------------------------------------------------------------------
def _acf(x: np.ndarray) -> np.ndarray:
    n = len(x)
    m = 1 << (2 * n - 1).bit_length()
    f = np.fft.rfft(x - x.mean(), n=m)
    r = np.fft.irfft(f * np.conj(f), n=m)[:n]
    return r / r[0] if r[0] > 0 else np.zeros(n)


def integrated_time(chain: np.ndarray, c: float = 5.0) -> np.ndarray:
    """tau per parameter for a (nsteps, nwalkers, ndim) chain: the
    walker-averaged autocorrelation function summed up to Sokal's automatic
    window (the smallest M with M >= c tau(M))."""
    nsteps, nw, d = chain.shape
    tau = np.empty(d)
    for k in range(d):
        f = np.mean([_acf(chain[:, w, k]) for w in range(nw)], axis=0)
        taus = 2.0 * np.cumsum(f) - 1.0
        m = np.arange(len(taus)) < c * taus
        win = int(np.argmin(m)) if not m.all() else len(taus) - 1
        tau[k] = taus[win]
    return tau


def ess(run: Run, burn: float = 0.25) -> tuple[float, np.ndarray]:
    """Minimum over parameters of (post-burn samples / tau), and the taus."""
    ch = run.chain[int(burn * run.chain.shape[0]):]
    tau = integrated_time(ch)
    n = ch.shape[0] * ch.shape[1]
    return float(np.min(n / tau)), tau


def posterior_summary(run: Run, burn: float = 0.25) -> dict:
    ch = run.chain[int(burn * run.chain.shape[0]):].reshape(-1, run.chain.shape[2])
    return {p: (float(ch[:, i].mean()), float(ch[:, i].std())) for i, p in enumerate(PARAMS)}


def initial_walkers(nwalkers: int, center: np.ndarray, seed: int, spread: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = center + spread * (PRIOR_HI - PRIOR_LO) * rng.standard_normal((nwalkers, len(center)))
    return np.clip(p, PRIOR_LO, PRIOR_HI)
