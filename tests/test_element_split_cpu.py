"""One model's element stage split into slabs across ranks, then its flux sum
split by time (sharded.light_curve_element_split), on CPU: two gloo ranks,
the oracle (the FP64 restatement of the reference's grid, eclipse and flux
code) standing in for the GPU engine as the element source.  Each rank
computes only its slab's records; the gathered element set, written into the
oracle's grids, must give the oracle's own unsplit light curve exactly (every
element's record is a function of that element alone, so the slab cut and the
gather order are the only things that can go wrong).
"""
import importlib
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

GRIDS = ("star1f", "star2f", "star1c", "star2c", "disc", "edge", "spot")
RECORD = np.dtype([("posn", "<f8", 3), ("dirn", "<f8", 3), ("area", "<f4"), ("gravity", "<f4"), ("flux", "<f4"),
                   ("necl", "<i4"), ("ecl", "<f8", 8)])


class OracleElements:
    """Element source over the oracle's grids, in the order of GRIDS; records
    as single uint8 rows of RECORD."""

    def __init__(self, text):
        from oracle import oracle as O
        self.O, self.text = O, text
        self.grids = O.Model(text=text).built_grids()
        self.sizes = [self.grids.fetch(g)["posn"].shape[0] for g in GRIDS]
        self.slabs_made = []

    def total(self):
        return sum(self.sizes)

    def slab(self, first, count):
        self.slabs_made.append((first, count))
        recs = np.zeros(self.total(), dtype=RECORD)
        at = 0
        for g, n in zip(GRIDS, self.sizes):
            d = self.grids.fetch(g)
            for k in RECORD.names:
                recs[k][at:at + n] = d[k]
            at += n
        return [torch.from_numpy(recs[first:first + count].view(np.uint8).reshape(count, RECORD.itemsize).copy())]

    def evaluate(self, arrays, shard):
        recs = arrays[0].numpy().reshape(-1).view(RECORD)
        assert recs.size == self.total()
        fresh = self.O.Model(text=self.text).built_grids()
        at = 0
        for g, n in zip(GRIDS, self.sizes):
            fresh.store(g, {k: recs[k][at:at + n] for k in RECORD.names})
            at += n
        o = fresh.light_curve(shard, scale=False, rdata=True)
        return o["calc"], {k: o[k] for k in ("wdwarf", "logg1", "logg2", "rv1", "rv2")}


def _case():
    W = importlib.import_module("lcurve-rs_b200.workloads")
    lcb = importlib.import_module("lcurve-rs_b200")
    text = W.single_large(nlat1=16, nlat2=30, ntime=10, nrad=16, nspot=20)[0]
    t = np.linspace(-0.2, 1.2, 97)
    d = lcb.make_data(t, expose=0.01, ndiv=3, ferr=0.01, weight=1.0)
    d["flux"] = 0.02 + 0.004 * np.cos(2 * np.pi * t)
    d["weight"][::11] = 0.0
    return text, d


def _run(group):
    from oracle import oracle as O
    S = importlib.import_module("lcurve-rs_b200.sharded")
    text, d = _case()
    out = []
    for scale in (True, False):
        src = OracleElements(text)
        r = S.light_curve_element_split(O.Model(text=text), d, scale=scale, group=group, source=src)
        out.append((r.calc, r.chisq, r.wnok, r.wdwarf, r.sfac, src.slabs_made))
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


def test_element_slabs_and_time_split_equal_the_unsplit_light_curve():
    from oracle import oracle as O
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    res = mp.Manager().dict()
    mp.spawn(_worker, args=(2, port, res), nprocs=2, join=True)
    text, d = _case()
    total = OracleElements(text).total()
    for k, scale in enumerate((True, False)):
        ref = O.Model(text=text).light_curve(d, scale=scale, rdata=True)
        for r in (0, 1):
            calc, chisq, wnok, wdwarf, sfac, slabs = res[r][k]
            # unscaled fluxes exactly; scaled ones through a re_scale summed in another order
            if scale:
                assert np.allclose(calc, ref["calc"], rtol=1e-12, atol=0), (scale, r)
            else:
                assert np.array_equal(calc, ref["calc"]), (scale, r)
            assert np.isclose(chisq, ref["chisq"], rtol=1e-12) and wnok == ref["wnok"]
            assert np.isclose(wdwarf, ref["wdwarf"], rtol=1e-12)
            assert np.allclose(sfac, ref["sfac"], rtol=1e-12)
        # each rank computed one half of the elements, and only that
        (f0, c0), = res[0][k][5]
        (f1, c1), = res[1][k][5]
        assert (f0, f0 + c0, f1 + c1) == (0, f1, total) and abs(c0 - c1) <= 1
