"""Work split across GPUs, one process per GPU (torch.distributed).

chisq_batch_sharded: one batch of models divided among the ranks by a cost
estimate (the reference's chisq_batch model loop, orchestration.rs:343-356),
each rank evaluating its models in one batch, the chi-squared all-gathered.

light_curve_sharded: one model's light curve split across GPUs by time.

The data (times) of a single large model are divided into contiguous shards,
one per rank of a torch.distributed process group (`mcmc.shard_bounds`).
Each rank evaluates the whole model (grids, eclipses, continuum) and the flux
sum for its own shard only, unscaled; the per-datum fluxes are all-gathered;
then every rank applies the reference's single-factor scaling and
chi-squared (orchestration.rs:264-310 with re_scale and compute_chisq,
orchestration.rs:361-401) to the full set, in FP64.  The flux sum, which
grows with elements x sub-phases, is divided among the ranks; the per-model
work is repeated on each.  Each datum's flux depends on its own time alone,
so the gathered fluxes are the unsplit evaluation's (to the flux sum's FP32
rounding, which depends on how the batch is cut into work units).

Models with per-component scale factors (iscale = 1) need the component
fluxes of every datum for their SVD fit and are not split here.
"""
from __future__ import annotations

import numpy as np

from . import DATUM_DTYPE, LcResult, Result
from .mcmc import _gather_rows, shard_bounds


def re_scale(data: np.ndarray, fit: np.ndarray) -> tuple[float, float, float]:
    """Single scale factor minimising chi-squared (orchestration.rs:361-389):
    returns (scale, chisq, wnok) and scales `fit` in place."""
    use = data["weight"] > 0.0
    wgt = data["weight"][use] / data["ferr"][use] ** 2
    sdy = float(np.sum(wgt * data["flux"][use] * fit[use]))
    syy = float(np.sum(wgt * fit[use] * fit[use]))
    wnok = float(np.sum(data["weight"][use]))
    if wnok > 0.0 and syy > 0.0:
        scale = sdy / syy
        fit *= scale
        chisq = float(np.sum(data["weight"][use] * ((data["flux"][use] - fit[use]) / data["ferr"][use]) ** 2))
        return scale, chisq, wnok
    return 1.0, 0.0, 0.0


def compute_chisq(data: np.ndarray, calc: np.ndarray) -> tuple[float, float]:
    """Weighted chi-squared and the weight sum (orchestration.rs:392-401)."""
    use = data["weight"] > 0.0
    chisq = float(np.sum(data["weight"][use] * ((data["flux"][use] - calc[use]) / data["ferr"][use]) ** 2))
    return chisq, float(np.sum(data["weight"][use]))


def _evaluate_engine(model, shard: np.ndarray):
    r = model.light_curve(data=shard, scale=False)
    return r.calc, dict(wdwarf=r.wdwarf, logg1=r.logg1, logg2=r.logg2, rv1=r.rv1, rv2=r.rv2)


def light_curve_sharded(model, data: np.ndarray, scale: bool = False, group=None, evaluate=None) -> LcResult:
    """Light curve of `model` at `data` (every rank passes the same) with the
    flux sum divided among the ranks of `group` (None: this process alone);
    returns what Model.light_curve(data=data, scale=scale) returns.

    evaluate(model, shard) -> (unscaled fluxes, {wdwarf, logg1, logg2, rv1,
    rv2}) computes one shard; by default the GPU engine through
    Model.light_curve."""
    data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
    if evaluate is None:
        if model.get_comp("iscale") not in ("0", "false"):
            raise ValueError("per-component scaling (iscale = 1) is not split across ranks")
        evaluate = _evaluate_engine
    n = data.shape[0]
    if group is None:
        calc, per_model = evaluate(model, data)
        calc = np.array(calc, dtype=np.float64)
    else:
        import torch.distributed as dist  # noqa: PLC0415
        b = shard_bounds(n, dist.get_world_size(group))
        r = dist.get_rank(group)
        local, per_model = evaluate(model, data[b[r]:b[r + 1]]) if b[r + 1] > b[r] else (np.zeros(0), None)
        if per_model is None:  # an empty shard still needs the model's own quantities
            _, per_model = evaluate(model, data[:1])
        calc = _gather_rows(np.asarray(local, dtype=np.float64), n, group)
    res = Result()
    res.logg1, res.logg2, res.rv1, res.rv2 = (per_model[k] for k in ("logg1", "logg2", "rv1", "rv2"))
    if scale:  # orchestration.rs:282-287
        s, res.chisq, res.wnok = re_scale(data, calc)
    else:      # orchestration.rs:300-309 (sfac = 1)
        s = 1.0
        res.chisq, res.wnok = compute_chisq(data, calc)
    res.wdwarf = per_model["wdwarf"] * s
    for k in range(5):
        res.sfac[k] = s
    return LcResult(data["time"], calc, res)


# ---------------------------------------------------------------------------
# One batch of models split across GPUs by cost (the reference's chisq_batch
# model loop, orchestration.rs:343-356, distributed over ranks)
# ---------------------------------------------------------------------------
# Device time per unit of work on a B200, measured on the 1024-model batch
# (k_flux, k_roche and k_elements stage times over their work counts), in
# units of one flux element-evaluation: an element eclipsed by a Roche-
# distorted star costs about 17,500 of them in the eclipse search, any grid
# element about 330 in the grid/continuum kernel.
ROCHE_WEIGHT = 17_500
ELEMENT_WEIGHT = 330


def model_costs(models, data: np.ndarray, offsets) -> np.ndarray:
    """Work estimate of each model of a ragged batch on its own data: flux
    element-evaluations + ROCHE_WEIGHT x Roche-eclipsed elements +
    ELEMENT_WEIGHT x grid elements (lcb_model_work: host planning only, no
    device work).  Physically invalid models cost 0."""
    from . import _capi  # noqa: PLC0415
    L = _capi.load()
    data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
    offs = np.asarray(offsets, dtype=np.int64)
    out = np.zeros(len(models))
    w = np.zeros(4, dtype=np.int64)
    for i, m in enumerate(models):
        lo, hi = int(offs[i]), int(offs[i + 1])
        _capi.check(L.lcb_model_work(m._h, data[lo:].ctypes.data, hi - lo, _capi.i64ptr(w)))
        out[i] = float(w[3]) + ROCHE_WEIGHT * float(w[1]) + ELEMENT_WEIGHT * float(w[0])
    return out


def partition(costs, world: int) -> list[np.ndarray]:
    """Models per rank: longest processing time first, each model to the rank
    with the least work so far (ties to the lower rank); every rank computes
    the same split.  Each rank's indices are returned in ascending order."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = np.zeros(costs.size, dtype=np.int64)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [np.flatnonzero(owner == r) for r in range(world)]


def _evaluate_batch_engine(models, data, offsets, scale):
    from . import chisq_batch_ragged  # noqa: PLC0415
    return chisq_batch_ragged(models, data, offsets, scale=scale)[0]


def chisq_batch_sharded(models, data: np.ndarray, offsets, scale: bool = False, group=None, evaluate=None,
                        costs=None) -> np.ndarray:
    """Chi-squared of every model of a ragged batch (model i on data[offsets[i]
    : offsets[i+1]]), the models divided among the ranks of `group` by cost
    (model_costs, partition); each rank evaluates its models in one batch and
    the per-model results are all-gathered, so every rank returns the whole
    batch's chi-squared (NaN for failed models, as chisq_batch_ragged).
    Every rank passes the same models, data and offsets.

    evaluate(models, data, offsets, scale) -> chisq evaluates one rank's
    share; by default the GPU engine (chisq_batch_ragged)."""
    data = np.ascontiguousarray(data, dtype=DATUM_DTYPE)
    offs = np.asarray(offsets, dtype=np.int64)
    n = len(models)
    evaluate = evaluate or _evaluate_batch_engine
    if group is None:
        return np.asarray(evaluate(list(models), data, offs, scale), dtype=np.float64)
    import torch  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    if costs is None:
        costs = model_costs(models, data, offs)
    parts = partition(costs, world)
    mine = parts[rank]
    local = np.zeros(0)
    if mine.size:
        sub = np.concatenate([data[offs[i]:offs[i + 1]] for i in mine])
        soffs = np.zeros(mine.size + 1, dtype=np.int64)
        soffs[1:] = np.cumsum([offs[i + 1] - offs[i] for i in mine])
        local = np.asarray(evaluate([models[i] for i in mine], sub, soffs, scale), dtype=np.float64)
    width = max(max(p.size for p in parts), 1)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.zeros(width, dtype=torch.float64, device=dev)
    buf[:local.size] = torch.as_tensor(local, dtype=torch.float64)
    got = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(got, buf, group=group)
    out = np.empty(n)
    for r in range(world):
        out[parts[r]] = got[r][:parts[r].size].cpu().numpy()
    return out


# ---------------------------------------------------------------------------
# One model's element stage split into slabs across GPUs, then its flux sum
# split by time (the grids and eclipse intervals of a ~5 M-element model are
# per-element work: crates/lcurve/src/grid.rs:227-320)
# ---------------------------------------------------------------------------
ELEMENT_ARRAYS = ("rec", "pos", "p64", "d64", "ecl")
ELEMENT_BYTES = (16, 16, 32, 32, 64)   # per element: float4, float4, double4, double4, 4 x double2


class EngineElements:
    """The GPU engine as an element source: slabs by lcb_model_elements into
    device tensors (uint8 rows of the records' bytes), light curves from a
    full element set by lcb_light_curve_elements."""

    def __init__(self, model):
        from . import _capi, _ctx  # noqa: PLC0415
        self.model, self._capi, self._ctx = model, _capi, _ctx
        self.L = _capi.load()

    def total(self) -> int:
        import ctypes as C  # noqa: PLC0415
        n = C.c_int64()
        self._capi.check(self.L.lcb_model_elements(self._ctx(), self.model._h, 0, 0, None, None, None, None, None,
                                                   C.byref(n)))
        return n.value

    def slab(self, first: int, count: int):
        import ctypes as C  # noqa: PLC0415
        import torch  # noqa: PLC0415
        dev = torch.device("cuda", torch.cuda.current_device())
        out = [torch.empty((max(count, 1), b), dtype=torch.uint8, device=dev) for b in ELEMENT_BYTES]
        torch.cuda.synchronize()
        n = C.c_int64()
        if count:
            self._capi.check(self.L.lcb_model_elements(self._ctx(), self.model._h, first, count,
                                                       *[C.c_void_p(t.data_ptr()) for t in out], C.byref(n)))
        return [t[:count] for t in out]

    def evaluate(self, arrays, shard: np.ndarray):
        import ctypes as C  # noqa: PLC0415
        import torch  # noqa: PLC0415
        from . import Result, dptr  # noqa: PLC0415
        shard = np.ascontiguousarray(shard, dtype=DATUM_DTYPE)
        arrays = [a.contiguous() for a in arrays]
        torch.cuda.synchronize()
        calc = np.zeros(shard.shape[0])
        res = Result()
        self._capi.check(self.L.lcb_light_curve_elements(self._ctx(), self.model._h, shard.ctypes.data,
                                                         shard.shape[0], 0, 1,
                                                         *[C.c_void_p(a.data_ptr()) for a in arrays],
                                                         dptr(calc), C.byref(res)))
        return calc, dict(wdwarf=res.wdwarf, logg1=res.logg1, logg2=res.logg2, rv1=res.rv1, rv2=res.rv2)


def _gather_records(local, counts, group):
    """All ranks' record slabs (per array: a (count, bytes) uint8 tensor) in
    rank order, concatenated; each array is sent padded to the largest slab."""
    import torch  # noqa: PLC0415
    import torch.distributed as dist  # noqa: PLC0415
    world = dist.get_world_size(group)
    width = max(max(counts), 1)
    out = []
    for a in local:
        buf = torch.zeros((width, a.shape[1]), dtype=torch.uint8, device=a.device)
        buf[:a.shape[0]] = a
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        out.append(torch.cat([parts[r][:counts[r]] for r in range(world)]))
    return out


def light_curve_element_split(model, data: np.ndarray, scale: bool = False, group=None, source=None) -> LcResult:
    """Light curve of one large model with both stages divided among the ranks
    of `group` (every rank passes the same model and data): the element list
    is cut into equal contiguous slabs (mcmc.shard_bounds), each rank computes
    its slab's grid points, continuum and eclipse intervals, the slabs are
    all-gathered into the full element set on every rank (each rank's own
    device memory; 160 B an element), and then the flux sum is split by time
    as light_curve_sharded does, every rank evaluating its share of the data
    from the gathered elements.  Returns what Model.light_curve(data=data,
    scale=scale) returns.

    source: the element source (total(), slab(first, count) -> per-array
    (count, bytes) uint8 tensors, evaluate(arrays, shard) -> (unscaled
    fluxes, {wdwarf, logg1, logg2, rv1, rv2})); by default the GPU engine."""
    if source is None:
        if model.get_comp("iscale") not in ("0", "false"):
            raise ValueError("per-component scaling (iscale = 1) is not split across ranks")
        source = EngineElements(model)
    total = source.total()
    if group is None:
        arrays = source.slab(0, total)
    else:
        import torch.distributed as dist  # noqa: PLC0415
        b = shard_bounds(total, dist.get_world_size(group))
        r = dist.get_rank(group)
        counts = [b[k + 1] - b[k] for k in range(len(b) - 1)]
        arrays = _gather_records(source.slab(b[r], counts[r]), counts, group)
    return light_curve_sharded(model, data, scale=scale, group=group,
                               evaluate=lambda m, shard: source.evaluate(arrays, shard))
