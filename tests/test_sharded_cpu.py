"""A single model's light curve split by time across ranks (sharded.py), on
CPU: two gloo ranks, each evaluating its shard of the data with the oracle
(the FP64 restatement of the reference path) standing in for the GPU engine;
the gathered, re-scaled result must equal the oracle's own unsplit
light_curve(scale=True / False): fluxes exactly (each datum's flux depends on
its time alone), chi-squared, weight sum, scale factors and wdwarf to 1e-12
(FP64 sums in another order).  Data include zero-weight points and an odd
count (uneven shards).
"""
import importlib
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import GOLDEN


def _data():
    lcb = importlib.import_module("lcurve-rs_b200")
    t = np.linspace(-0.2, 1.2, 301)
    d = lcb.make_data(t, expose=0.001, ndiv=1, ferr=0.01, weight=1.0)
    d["flux"] = 0.02 + 0.005 * np.cos(2 * np.pi * t)
    d["weight"][::17] = 0.0
    d["ndiv"][::5] = 3
    return d


def _evaluate(om, shard):
    out = om.light_curve(shard, scale=False, rdata=True)
    return out["calc"], {k: out[k] for k in ("wdwarf", "logg1", "logg2", "rv1", "rv2")}


def _run(group):
    from oracle import oracle as O
    S = importlib.import_module("lcurve-rs_b200.sharded")
    om = O.Model(GOLDEN / "test_model.dat")
    out = []
    for scale in (True, False):
        r = S.light_curve_sharded(om, _data(), scale=scale, group=group, evaluate=_evaluate)
        out.append((r.calc, r.chisq, r.wnok, r.wdwarf, r.sfac, r.logg1, r.rv2))
    return out


def _worker(rank, world, port, res):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res[rank] = _run(dist.group.WORLD)
    finally:
        dist.destroy_process_group()


def test_time_split_light_curve_equals_the_unsplit_one():
    from oracle import oracle as O
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    res = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, res), nprocs=2, join=True)
    om = O.Model(GOLDEN / "test_model.dat")
    for k, scale in enumerate((True, False)):
        ref = om.light_curve(_data(), scale=scale, rdata=True)
        for rank in (0, 1):
            calc, chisq, wnok, wdwarf, sfac, logg1, rv2 = res[rank][k]
            assert np.allclose(calc, ref["calc"], rtol=1e-12, atol=0)
            assert np.isclose(chisq, ref["chisq"], rtol=1e-12) and wnok == ref["wnok"]
            assert np.isclose(wdwarf, ref["wdwarf"], rtol=1e-12)
            assert np.allclose(sfac, ref["sfac"][:5] if scale else np.ones(5), rtol=1e-12)
            assert logg1 == ref["logg1"] and rv2 == ref["rv2"]
    # this process alone gives the same
    alone = _run(None)
    assert np.array_equal(alone[0][0], res[0][0][0])
