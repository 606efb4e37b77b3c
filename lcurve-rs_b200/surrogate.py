"""Light-curve surrogate: training data from the GPU engine, a BF16
tensor-core MLP trained on it, and fast surrogate chi-squared.

The network (lcurve_b200_surrogate.h) maps the five fitted parameters
(q, iangle, r1 and the two stars' Planck exponents h c / lambda k T, each
scaled to [-1, 1] over the prior box) to the shape
of the light curve on a fixed phase grid (natural-log fluxes minus their
mean, centred per phase and scaled by one global factor).
Curves for training come from the light-curve engine itself (resident
batches, lcurve_b200.h), so the surrogate's error is measured against the
method it stands in for.  Device buffers are torch tensors (plumbing only);
every arithmetic kernel of training and inference is the library's own.

The reference has no surrogate; the likelihood it approximates is the
reference fitter's -chisq/2 with chisq from chisq_batch(scale=True)
(python/lcurve_rs/fitting.py:285-341, crates/lcurve/src/orchestration.rs:329-401).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import time

import numpy as np

from . import Batch, Model, _capi, make_data
from . import workloads as W

PARAMS = ("q", "iangle", "r1", "t1", "t2")
PRIOR_LO = np.array([0.05, 75.0, 0.005, 8000.0, 2500.0])
PRIOR_HI = np.array([1.0, 90.0, 0.03, 40000.0, 5000.0])
TRUTH = np.array([0.5, 82.0, 0.015, 15000.0, 3500.0])


HC_OVER_LK = 1.4387769e7 / 550.0   # h c / (lambda k) in K at the model's 550 nm


def features(theta: np.ndarray) -> np.ndarray:
    """Network inputs: q, iangle, r1 and the Planck exponents h c / (lambda k T)
    of the two stars (the temperatures enter the fluxes through them)."""
    x = np.array(theta, dtype=np.float64, copy=True, ndmin=2)
    x[:, 3] = HC_OVER_LK / x[:, 3]
    x[:, 4] = HC_OVER_LK / x[:, 4]
    return x


_F = features(np.vstack([PRIOR_LO, PRIOR_HI]))
FEAT_LO, FEAT_HI = _F.min(axis=0), _F.max(axis=0)


def _torch():
    import torch  # noqa: PLC0415 - device memory and streams only

    return torch


@dataclasses.dataclass
class CurveSetup:
    """The fixed model and phase grid the surrogate learns: the 15,926-element
    single-star-pair model (nlat1f=50, nlat2f=100, Claret WD, Roche-filling
    secondary) at n_phase phases uniform in [-0.2, 0.8]."""

    n_phase: int = 256
    expose: float = 0.001
    ndiv: int = 1

    @property
    def text(self) -> str:
        return W.model_text(**W.SMALL)

    @property
    def times(self) -> np.ndarray:
        return np.linspace(-0.2, 0.8, self.n_phase)


def sample_prior(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return PRIOR_LO + (PRIOR_HI - PRIOR_LO) * rng.random((n, len(PARAMS)))


class CurveEngine:
    """Resident batches of the setup's model for a few batch sizes; evaluates
    (N x 5) parameter rows to light curves or chi-squared against data."""

    def __init__(self, setup: CurveSetup, data: np.ndarray | None = None,
                 sizes=(4, 8, 12, 16, 24, 32, 48, 64, 96, 128)):
        self.setup = setup
        base = Model(text=setup.text)
        if data is None:
            data = make_data(setup.times, expose=setup.expose, ndiv=setup.ndiv, ferr=1.0, weight=1.0)
        self.data = data
        self.sizes = tuple(sorted(sizes))
        self._batches = {}
        self._base = base
        self.evals = 0

    def _batch(self, size: int) -> Batch:
        b = self._batches.get(size)
        if b is None:
            nd = self.data.shape[0]
            models = [self._base] * size
            data = np.concatenate([self.data] * size)
            b = Batch(models, data, np.arange(size + 1, dtype=np.int64) * nd)
            self._batches[size] = b
        return b

    def _run(self, theta: np.ndarray, scale: bool, want_calc: bool):
        theta = np.atleast_2d(np.asarray(theta, dtype=np.float64))
        n = theta.shape[0]
        size = next((s for s in self.sizes if s >= n), None)
        if size is None:
            raise ValueError(f"at most {self.sizes[-1]} rows per call")
        pad = np.concatenate([theta, np.repeat(theta[-1:], size - n, axis=0)]) if size > n else theta
        b = self._batch(size)
        b.set_params(PARAMS, pad)
        b.run(scale=scale)
        self.evals += n
        if not want_calc:
            return b.chisq()[:n], None
        chisq, calc, _ = b.results(want_calc=True)
        return chisq[:n], calc.reshape(size, -1)[:n]

    def chisq(self, theta: np.ndarray, scale: bool = True) -> np.ndarray:
        return self._run(theta, scale, False)[0]

    def curves(self, theta: np.ndarray) -> np.ndarray:
        """(N x n_phase) model fluxes; rows of failed models are NaN."""
        chisq, calc = self._run(theta, False, True)
        calc = calc.copy()
        calc[~np.isfinite(chisq)] = np.nan
        return calc


def generate_curves(setup: CurveSetup, theta: np.ndarray, chunk: int = 4096, log=None) -> np.ndarray:
    """Light curves of every parameter row, in resident batches of `chunk` models."""
    eng = CurveEngine(setup, sizes=(chunk,))
    out = np.empty((theta.shape[0], setup.n_phase))
    t0 = time.perf_counter()
    for i in range(0, theta.shape[0], chunk):
        out[i:i + chunk] = eng.curves(theta[i:i + chunk])
        if log and (i // chunk) % 32 == 0:
            log(f"curves {i + chunk}/{theta.shape[0]} in {time.perf_counter() - t0:.1f} s")
    return out


def shard_rows(k: int, batch: int, rank: int, world: int) -> slice:
    """Rows of the k-th global batch (of `batch` rows, a multiple of `world`)
    that data-parallel rank `rank` trains on: equal contiguous shards."""
    local = batch // world
    return slice(k * batch + rank * local, k * batch + (rank + 1) * local)


def _shape(flux: np.ndarray) -> np.ndarray:
    lf = np.log(flux)
    return lf - lf.mean(axis=1, keepdims=True)


def scaled_rel_error(pred: np.ndarray, flux: np.ndarray) -> np.ndarray:
    """|s pred - flux| / flux per point, s the least-squares scale of each row
    (the comparison the scale-fitted likelihood makes)."""
    s = np.sum(pred * flux, axis=1, keepdims=True) / np.sum(pred * pred, axis=1, keepdims=True)
    return np.abs(s * pred - flux) / np.abs(flux)


class Surrogate:
    """The MLP, its input/output normalisation, training and inference."""

    def __init__(self, n_phase: int = 256, width: int = 512, n_hidden: int = 4, max_batch: int = 8192, seed: int = 0,
                 device: int = 0, box: tuple | None = None):
        """box = (lo, hi): the parameter box the inputs are scaled to [-1, 1]
        over (default the prior box); a local surrogate uses a small one.
        Proposals outside the prior box are rejected either way."""
        torch = _torch()
        self.L = _capi.load()
        self.n_phase, self.width, self.n_hidden = n_phase, width, n_hidden
        self.max_batch = max_batch
        self.dev = torch.device("cuda", device)
        self._h = C.c_void_p()
        _capi.check_mlp(self.L.lcb_mlp_create(device, len(PARAMS), width, n_hidden, n_phase, max_batch, seed,
                                              C.byref(self._h)))
        self._stream = torch.cuda.Stream(device=self.dev)
        _capi.check_mlp(self.L.lcb_mlp_set_stream(self._h, C.c_void_p(self._stream.cuda_stream)))
        self.mean = torch.zeros(n_phase, dtype=torch.float32, device=self.dev)
        self.sd = torch.ones(n_phase, dtype=torch.float32, device=self.dev)
        self._y = torch.empty(max_batch, n_phase, dtype=torch.float32, device=self.dev)
        self.train_seconds = 0.0
        # the same input map for the device sub-chain: fadd + fmul * (x or 1/x)
        d = len(PARAMS)
        recip = [0, 0, 0, 1, 1]
        self.box = (np.array(PRIOR_LO), np.array(PRIOR_HI)) if box is None else (np.array(box[0]), np.array(box[1]))
        f = features(np.vstack(self.box))
        flo, fhi = f.min(axis=0), f.max(axis=0)
        span = fhi - flo
        self._c_lo = (C.c_double * d)(*PRIOR_LO)
        self._c_hi = (C.c_double * d)(*PRIOR_HI)
        self._c_recip = (C.c_int * d)(*recip)
        self._c_fmul = (C.c_float * d)(*[2.0 / span[k] * (HC_OVER_LK if recip[k] else 1.0) for k in range(d)])
        self._c_fadd = (C.c_float * d)(*[-2.0 * flo[k] / span[k] - 1.0 for k in range(d)])
        self._recip = np.array(recip, dtype=bool)
        self._fmul64 = np.array(self._c_fmul, dtype=np.float32).astype(np.float64)
        self._fadd64 = np.array(self._c_fadd, dtype=np.float32).astype(np.float64)

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_capi, "_lib", None) if _capi is not None else None  # None at interpreter exit
        if h and lib is not None:
            lib.lcb_mlp_destroy(h)
            self._h = None

    def _x(self, theta):
        """Network inputs, computed exactly as the device sub-chain computes
        them: fadd + fmul * (x or 1/x) in double precision, rounded once to
        float (the network then rounds them to bfloat16)."""
        torch = _torch()
        th = np.array(theta, dtype=np.float64, ndmin=2)
        with np.errstate(divide="ignore", invalid="ignore"):
            f = np.where(self._recip, 1.0 / th, th)
        x = (self._fadd64 + self._fmul64 * f).astype(np.float32)
        return torch.as_tensor(x).to(self.dev)

    def fit(self, theta: np.ndarray, flux: np.ndarray, epochs: int = 60, batch: int = 8192, lr: float = 2e-3,
            lr_min: float = 2e-5, log=None, group=None, renormalize: bool = True) -> list[float]:
        """Trains on (theta, flux) rows with finite fluxes; cosine learning-rate
        schedule, Adam.  Returns the mean training loss of each epoch.

        The target is the curve's shape, ln f_j minus the curve's mean ln f:
        the likelihood it serves fits the flux scale per model (scale=True),
        so the overall level carries no information and is not learned.

        group: a torch.distributed process group (one rank per GPU, every rank
        with the same data, seed and arguments) for data-parallel training:
        each global batch is split into equal contiguous shards, one per rank
        (shard_rows), and the ranks' gradients are averaged by an all-reduce on
        the network's stream before the Adam step, so every rank takes the
        step of the whole batch and the weights stay identical.  The returned
        losses are this rank's shards'."""
        torch = _torch()
        rank, world = 0, 1
        if group is not None:
            import torch.distributed as dist  # noqa: PLC0415
            rank, world = dist.get_rank(group), dist.get_world_size(group)
        ok = np.all(np.isfinite(flux), axis=1) & np.all(flux > 0, axis=1)
        theta, flux = theta[ok], flux[ok]
        with torch.cuda.stream(self._stream):
            logf = torch.as_tensor(_shape(flux), dtype=torch.float32).to(self.dev)
            # one scale for every phase: the loss is then the mean squared
            # log-flux error, the quantity the chi-squared weighs uniformly;
            # a further fit (renormalize=False) keeps the trained network's scale
            if renormalize:
                self.mean = logf.mean(dim=0)
                self.sd = torch.full_like(self.mean, float((logf - self.mean).std().clamp_min(1e-6)))
            Y = ((logf - self.mean) / self.sd).contiguous()
            X = self._x(theta)
        self._stream.synchronize()
        n = X.shape[0]
        local = min(batch // world, self.max_batch, (n // world) - (n // world) % 8)
        local -= local % 8
        if local <= 0:
            raise ValueError("too few rows for one batch of 8 per rank")
        batch = local * world
        steps_per_epoch = n // batch
        grads = self._grads_tensor() if group is not None else None
        total = epochs * steps_per_epoch
        g = torch.Generator(device=self.dev).manual_seed(0)
        losses = []
        step = 0
        t0 = time.perf_counter()
        for ep in range(epochs):
            with torch.cuda.stream(self._stream):
                perm = torch.randperm(n, device=self.dev, generator=g)
            for k in range(steps_per_epoch):
                rate = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * step / max(total, 1)))
                with torch.cuda.stream(self._stream):
                    idx = perm[shard_rows(k, batch, rank, world)]
                    xb = X.index_select(0, idx)
                    yb = Y.index_select(0, idx)
                if group is None:
                    _capi.check_mlp(self.L.lcb_mlp_train_step(self._h, C.c_void_p(xb.data_ptr()),
                                                              C.c_void_p(yb.data_ptr()), local, rate, 0.9, 0.999,
                                                              1e-8, 0.0))
                else:
                    _capi.check_mlp(self.L.lcb_mlp_backward(self._h, C.c_void_p(xb.data_ptr()),
                                                            C.c_void_p(yb.data_ptr()), local))
                    with torch.cuda.stream(self._stream):  # ordered after the backward, before the step
                        dist.all_reduce(grads, group=group)
                        grads.div_(world)
                    _capi.check_mlp(self.L.lcb_mlp_adam_step(self._h, rate, 0.9, 0.999, 1e-8, 0.0))
                step += 1
            v = C.c_double()
            _capi.check_mlp(self.L.lcb_mlp_take_loss(self._h, C.byref(v)))
            losses.append(v.value / steps_per_epoch)
            if log and (ep % 10 == 0 or ep == epochs - 1):
                log(f"epoch {ep} loss {losses[-1]:.3e} ({time.perf_counter() - t0:.1f} s)")
        self.train_seconds += time.perf_counter() - t0
        return losses

    def save(self, path) -> None:
        """Checkpoint (.npz): the network's shape, its training state (FP32
        parameters, Adam moments and step count), the output normalisation and
        the training time so far.  Surrogate.load resumes training exactly."""
        n = C.c_int64()
        _capi.check_mlp(self.L.lcb_mlp_state_size(self._h, C.byref(n)))
        state = np.empty(3 * n.value, dtype=np.float32)
        steps = C.c_int64()
        _capi.check_mlp(self.L.lcb_mlp_get_state(self._h, C.c_void_p(state.ctypes.data), state.size,
                                                 C.byref(steps)))
        np.savez(path, state=state, steps=steps.value, mean=self.mean.cpu().numpy(), sd=self.sd.cpu().numpy(),
                 shape=np.array([self.n_phase, self.width, self.n_hidden, self.max_batch]),
                 train_seconds=self.train_seconds, box=np.vstack(self.box))

    @classmethod
    def load(cls, path, device: int = 0) -> "Surrogate":
        torch = _torch()
        with np.load(path) as z:
            n_phase, width, n_hidden, max_batch = (int(v) for v in z["shape"])
            sur = cls(n_phase=n_phase, width=width, n_hidden=n_hidden, max_batch=max_batch, device=device,
                      box=tuple(z["box"]) if "box" in z.files else None)
            state = np.ascontiguousarray(z["state"], dtype=np.float32)
            _capi.check_mlp(sur.L.lcb_mlp_set_state(sur._h, C.c_void_p(state.ctypes.data), state.size,
                                                    int(z["steps"])))
            sur.mean = torch.as_tensor(z["mean"]).to(sur.dev)
            sur.sd = torch.as_tensor(z["sd"]).to(sur.dev)
            sur.train_seconds = float(z["train_seconds"])
        return sur

    def _grads_tensor(self):
        """The network's device gradient buffer as a torch tensor (no copy)."""
        torch = _torch()
        ptr, n = C.POINTER(C.c_float)(), C.c_int64()
        _capi.check_mlp(self.L.lcb_mlp_grads_device(self._h, C.byref(ptr), C.byref(n)))

        class _View:  # __cuda_array_interface__ of the library-owned buffer
            __cuda_array_interface__ = {"shape": (n.value,), "typestr": "<f4", "version": 2,
                                        "data": (C.cast(ptr, C.c_void_p).value, False), "strides": None}

        return torch.as_tensor(_View(), device=self.dev)

    def _forward_dev(self, X):
        n = X.shape[0]
        if n > self.max_batch:
            raise ValueError("too many rows")
        _capi.check_mlp(self.L.lcb_mlp_forward(self._h, C.c_void_p(X.data_ptr()), n, C.c_void_p(self._y.data_ptr())))
        return self._y[:n]

    def predict(self, theta: np.ndarray) -> np.ndarray:
        """(N x n_phase) surrogate fluxes, up to a constant factor per curve
        (exp of the predicted shape)."""
        torch = _torch()
        theta = np.atleast_2d(theta)
        out = np.empty((theta.shape[0], self.n_phase))
        for i in range(0, theta.shape[0], self.max_batch):
            with torch.cuda.stream(self._stream):
                y = self._forward_dev(self._x(theta[i:i + self.max_batch]))
                f = torch.exp(y.double() * self.sd.double() + self.mean.double())
                out[i:i + self.max_batch] = f.cpu().numpy()
        return out

    def bind_data(self, data: np.ndarray) -> None:
        """Data (make_data records on the setup's phase grid) for chisq()."""
        torch = _torch()
        self._flux = torch.as_tensor(np.ascontiguousarray(data["flux"]), dtype=torch.float64).to(self.dev)
        self._ferr = torch.as_tensor(np.ascontiguousarray(data["ferr"]), dtype=torch.float64).to(self.dev)
        self._chi = torch.empty(self.max_batch, dtype=torch.float64, device=self.dev)

    def chisq(self, theta: np.ndarray, scale: bool = True) -> np.ndarray:
        """Surrogate chi-squared of each row against the bound data (one
        forward pass and one reduction kernel)."""
        torch = _torch()
        theta = np.atleast_2d(theta)
        n = theta.shape[0]
        with torch.cuda.stream(self._stream):
            y = self._forward_dev(self._x(theta))
            _capi.check_mlp(self.L.lcb_logflux_chisq(n, self.n_phase, C.c_void_p(y.data_ptr()),
                                                     C.c_void_p(self.mean.data_ptr()), C.c_void_p(self.sd.data_ptr()),
                                                     C.c_void_p(self._flux.data_ptr()),
                                                     C.c_void_p(self._ferr.data_ptr()), int(bool(scale)),
                                                     C.c_void_p(self._chi.data_ptr()), C.c_void_p(self._stream.cuda_stream)))
            out = self._chi[:n].cpu().numpy()
        return out

    def subchain(self, y: np.ndarray, ls: np.ndarray, comp: np.ndarray, rnd: np.ndarray, a: float = 2.0,
                 scale: bool = True, move: str = "stretch", bandwidth: float = 1.0):
        """Runs rnd.shape[0] surrogate Metropolis moves (stretch or KDE) of the
        walkers y (log probabilities ls) against the fixed walkers comp on the
        device (lcb_surrogate_subchain_host); returns the new (y, ls)."""
        from .mcmc import KDE  # noqa: PLC0415
        y = np.ascontiguousarray(y, dtype=np.float64)
        n, d = y.shape
        if move == "kde":
            kde = KDE.of(np.asarray(comp, dtype=np.float64), bandwidth)
            keep = (np.ascontiguousarray(kde.chol), np.ascontiguousarray(kde.prec))  # alive through the call
            chol = keep[0].ctypes.data_as(C.POINTER(C.c_double))
            prec = keep[1].ctypes.data_as(C.POINTER(C.c_double))
        else:
            chol = prec = None
            keep = ()
        comp = np.ascontiguousarray(comp, dtype=np.float64)
        m = comp.shape[0]
        y = y.copy()
        ls = np.array(ls, dtype=np.float64)
        rnd = np.ascontiguousarray(rnd, dtype=np.float64)
        # host arrays in and out: the library stages them through its own page-locked buffer
        _capi.check_mlp(self.L.lcb_surrogate_subchain_host(
            self._h, n, m, d, y.ctypes.data, ls.ctypes.data, comp.ctypes.data, rnd.ctypes.data, rnd.shape[0], a,
            self._c_lo, self._c_hi, self._c_recip, self._c_fmul, self._c_fadd, C.c_void_p(self.mean.data_ptr()),
            C.c_void_p(self.sd.data_ptr()), C.c_void_p(self._flux.data_ptr()), C.c_void_p(self._ferr.data_ptr()),
            int(bool(scale)), 1 if move == "kde" else 0, chol, prec))
        del keep
        return y, ls


def refine_near(sur: Surrogate, setup: CurveSetup, ensemble: np.ndarray, theta_global: np.ndarray,
                flux_global: np.ndarray, n: int = 131072, widen: float = 3.0, epochs: int = 40, seed: int = 7,
                lr: float = 5e-4, log=None) -> float:
    """Sharpens the surrogate where a sampler's ensemble sits: n parameter
    rows drawn from a Gaussian with the ensemble's mean and covariance widened
    by `widen` (kept inside the prior box), their curves computed by the
    engine, and `epochs` further epochs of training on them mixed with as
    many rows of the global training set (so the rest of the box is kept).
    The sampler that uses the surrogate afterwards stays exact: delayed
    acceptance corrects any surrogate error, a better surrogate only wastes
    fewer engine evaluations.  Returns the seconds spent (curves + training)."""
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    mu = ensemble.mean(axis=0)
    cov = np.cov(ensemble, rowvar=False) * widen ** 2 + np.diag(1e-12 * (PRIOR_HI - PRIOR_LO) ** 2)
    local = rng.multivariate_normal(mu, cov, size=2 * n)
    local = local[np.all((local >= PRIOR_LO) & (local <= PRIOR_HI), axis=1)][:n]
    curves = generate_curves(setup, local)
    pick = rng.choice(theta_global.shape[0], size=min(n, theta_global.shape[0]), replace=False)
    theta = np.concatenate([local, theta_global[pick]])
    flux = np.concatenate([curves, flux_global[pick]])
    sur.fit(theta, flux, epochs=epochs, lr=lr, lr_min=lr * 0.01, log=log, renormalize=False)
    return time.perf_counter() - t0


def local_surrogate(setup: CurveSetup, ensemble: np.ndarray, n: int = 262144, widen: float = 4.0,
                    epochs: int = 200, seed: int = 11, data=None, log=None) -> tuple["Surrogate", float]:
    """A second network for where a sampler's ensemble sits: trained from
    scratch on n engine curves drawn from a Gaussian with the ensemble's mean
    and covariance widened by `widen` (inside the prior box), its inputs
    scaled over that region (the ensemble's range widened likewise), so the
    same network resolves the curve's small variations there.  The sampler
    that uses it stays exact (delayed acceptance), and it still rejects
    proposals outside the prior box.  Returns (surrogate, seconds)."""
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    mu = ensemble.mean(axis=0)
    cov = np.cov(ensemble, rowvar=False) * widen ** 2 + np.diag(1e-12 * (PRIOR_HI - PRIOR_LO) ** 2)
    theta = rng.multivariate_normal(mu, cov, size=2 * n)
    theta = theta[np.all((theta >= PRIOR_LO) & (theta <= PRIOR_HI), axis=1)][:n]
    lo, hi = theta.min(axis=0), theta.max(axis=0)
    curves = generate_curves(setup, theta)
    sur = Surrogate(box=(lo, hi))
    sur.fit(theta, curves, epochs=epochs, log=log)
    if data is not None:
        sur.bind_data(data)
    return sur, time.perf_counter() - t0
