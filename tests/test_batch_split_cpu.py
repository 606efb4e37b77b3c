"""One ragged batch split across ranks by cost (sharded.chisq_batch_sharded),
on CPU: two gloo ranks, each evaluating its share of the models with the
oracle (the FP64 restatement of the reference's chisq_batch model loop,
orchestration.rs:343-356) standing in for the GPU engine; the all-gathered
chi-squared must equal the oracle's unsplit chisq_ragged exactly (each
model's chi-squared depends on that model alone).  The cost split itself:
every model assigned once, loads balanced, the same on every rank.
"""
import importlib
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _batch():
    W = importlib.import_module("lcurve-rs_b200.workloads")
    lcb = importlib.import_module("lcurve-rs_b200")
    specs = W.batch_models(n=7, seed=21, nlat1=(10, 30), nlat2=(10, 40), ntime=(40, 120))
    offs = np.zeros(len(specs) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(t) for _, t in specs])
    times = np.concatenate([t for _, t in specs])
    data = lcb.make_data(times, expose=0.001, ndiv=1, flux=1.0, ferr=0.05, weight=1.0)
    data["flux"] = 0.02 + 0.004 * np.cos(2 * np.pi * times)
    return specs, data, offs


def _evaluate(oms, data, offs, scale):
    from oracle import oracle as O
    return O.chisq_ragged(oms, data, offs, scale=scale, nthreads=2)


def _run(group):
    from oracle import oracle as O
    lcb = importlib.import_module("lcurve-rs_b200")
    S = importlib.import_module("lcurve-rs_b200.sharded")
    specs, data, offs = _batch()
    costs = S.model_costs([lcb.Model(text=s) for s, _ in specs], data, offs)
    oms = [O.Model(text=s) for s, _ in specs]
    return [S.chisq_batch_sharded(oms, data, offs, scale=sc, group=group, evaluate=_evaluate, costs=costs)
            for sc in (False, True)], costs


def _worker(rank, world, port, res):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res[rank] = _run(dist.group.WORLD)
    finally:
        dist.destroy_process_group()


def test_batch_split_by_cost_equals_the_unsplit_batch():
    from oracle import oracle as O
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    res = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, res), nprocs=2, join=True)
    specs, data, offs = _batch()
    oms = [O.Model(text=s) for s, _ in specs]
    for k, sc in enumerate((False, True)):
        ref = O.chisq_ragged(oms, data, offs, scale=sc, nthreads=2)
        assert np.all(np.isfinite(ref))
        for r in (0, 1):
            assert np.array_equal(res[r][0][k], ref), (sc, r)
    assert np.array_equal(res[0][1], res[1][1])  # both ranks weigh the models alike


def test_cost_partition_is_complete_and_balanced():
    S = importlib.import_module("lcurve-rs_b200.sharded")
    rng = np.random.default_rng(3)
    costs = rng.lognormal(0.0, 1.0, 1024)
    for world in (1, 2, 3, 8):
        parts = S.partition(costs, world)
        assert sorted(np.concatenate(parts).tolist()) == list(range(costs.size))
        loads = np.array([costs[p].sum() for p in parts])
        assert loads.max() <= costs.sum() / world + costs.max()  # greedy bound
        assert loads.max() / loads.mean() < 1.02
        assert all(np.all(np.diff(p) > 0) for p in parts)


def test_model_costs_follow_the_work():
    lcb = importlib.import_module("lcurve-rs_b200")
    S = importlib.import_module("lcurve-rs_b200.sharded")
    W = importlib.import_module("lcurve-rs_b200.workloads")
    small, big = W.model_text(nlat1f=20, nlat2f=40), W.model_text(nlat1f=60, nlat2f=120)
    t = np.linspace(-0.2, 1.2, 100)
    d = lcb.make_data(np.concatenate([t, t]), ferr=1.0)
    c = S.model_costs([lcb.Model(text=small), lcb.Model(text=big)], d, [0, 100, 200])
    assert 0 < c[0] < c[1]
    bad = lcb.Model(text=W.model_text(r2=0.99, roche2=0))  # larger than its Roche lobe: no work
    assert S.model_costs([bad], d[:100], [0, 100])[0] == 0.0
