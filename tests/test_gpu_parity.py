"""GPU parity: the CUDA path through the C ABI against the CPU oracle and the
reference's golden vectors.  Tolerance: max relative error 1e-5 on fluxes
(the FP32 flux sum with compensated accumulation against the FP64 oracle).
"""
import importlib

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def W():
    return importlib.import_module("lcurve-rs_b200.workloads")


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def gpu_and_oracle_lc(lcb, oracle, text, times, expose, ndiv, scale=False, rdata=False, data=None):
    d = data if data is not None else lcb.make_data(times, expose=expose, ndiv=ndiv, ferr=1.0, weight=1.0)
    m = lcb.Model(text=text)
    calc = np.zeros(d.shape[0])
    import ctypes as C
    res = lcb.Result()
    lcb._capi.check(lcb._capi.load().lcb_light_curve(lcb._ctx(), m._h, d.ctypes.data, d.shape[0], int(scale),
                                                     int(rdata), lcb._capi.dptr(calc), C.byref(res)))
    o = oracle.Model(text=text).light_curve(d, scale=scale, rdata=rdata, nthreads=8)
    return calc, res, o


def test_golden_cpp_light_curve(lcb):
    m = lcb.Model(GOLDEN / "test_model.dat")
    r = m.light_curve(time1=-0.2, time2=1.2, ntime=500, expose=0.001, ndiv=1)
    g = np.loadtxt(GOLDEN / "test_lc.dat")
    assert rel_err(r.flux, g[:, 2]) < TOL
    assert np.array_equal(r.times, g[:, 0])


def test_golden_model_matches_oracle_scalars(lcb, oracle):
    text = (GOLDEN / "test_model.dat").read_text()
    t = np.linspace(-0.2, 1.2, 500)
    calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, 0.001, 1)
    assert rel_err(calc, o["calc"]) < TOL
    assert abs(res.wdwarf - o["wdwarf"]) <= 1e-9 * abs(o["wdwarf"])
    assert abs(res.rv1 - o["rv1"]) < 1e-12 and abs(res.rv2 - o["rv2"]) < 1e-12
    assert res.logg1 == o["logg1"] and res.logg2 == o["logg2"]


def test_single_small_vs_oracle(lcb, oracle, W):
    text, t, expose, ndiv = W.single_small()
    calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, expose, ndiv)
    assert rel_err(calc, o["calc"]) < TOL


def test_disc_edge_spot_irradiation_vs_oracle(lcb, oracle, W):
    text, t, expose, ndiv = W.single_large(nlat1=40, nlat2=80, ntime=1500, nrad=50, nspot=40)
    calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, expose, ndiv)
    assert rel_err(calc, o["calc"]) < TOL
    assert abs(res.wdwarf - o["wdwarf"]) <= 1e-7 * abs(o["wdwarf"])


def test_lensing_spots_vs_oracle(lcb, oracle, W):
    text, t, expose, ndiv = W.single_huge(nlat1=40, nlat2=80, ntime=800, nrad=50)
    calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, expose, ndiv)
    assert rel_err(calc, o["calc"]) < TOL


def test_beaming_and_coarse_grids_vs_oracle(lcb, oracle, W):
    text = W.model_text(velocity_scale=300.0, beam_factor1=1.3, beam_factor2=0.8, spin1=1.1, spin2=0.9,
                        nlat1f=40, nlat1c=20, nlat2f=60, nlat2c=30, limb1="Claret", ldc1_1=0.5, ldc1_2=-0.2,
                        ldc1_3=0.3, ldc1_4=-0.1, mucrit1=0.01)
    t = np.linspace(-0.3, 1.3, 700)
    calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, 0.003, 3)
    assert rel_err(calc, o["calc"]) < TOL
    assert abs(res.wdwarf - o["wdwarf"]) <= 1e-7 * abs(o["wdwarf"])


def test_light_curve_scale_and_chisq(lcb, oracle, W):
    text, t, expose, ndiv = W.single_small()
    base = lcb.Model(text=text).light_curve(times=t, expose=expose, ndiv=ndiv).flux
    d = W.noisy_data(t, 2.5 * base, expose, ndiv, seed=3)
    for scale in (False, True):
        calc, res, o = gpu_and_oracle_lc(lcb, oracle, text, t, expose, ndiv, scale=scale, rdata=True, data=d)
        assert rel_err(calc, o["calc"]) < TOL
        assert abs(res.chisq - o["chisq"]) <= 1e-4 * abs(o["chisq"])
        assert res.wnok == o["wnok"]
        assert np.allclose(list(res.sfac), o["sfac"], rtol=1e-5)


def test_chisq_batch_vs_oracle(lcb, oracle):
    # tests/chisq_batch.rs and crates/lcurve-cuda/tests/gpu_correctness.rs shapes
    text = (GOLDEN / "test_model.dat").read_text()
    t = np.linspace(-0.2, 1.2, 200)
    d = lcb.make_data(t, expose=0.001, ndiv=1, flux=1.0e-9, ferr=1.0e-11, weight=1.0)
    n = 16
    frac = np.arange(n) / (n - 1) - 0.5
    vals = np.stack([0.5 + 0.02 * frac, 82.0 + 2.0 * frac], axis=1)
    m = lcb.Model(text=text)
    o = oracle.Model(text=text)
    for scale in (False, True):
        g = m.chisq_batch(d, ["q", "iangle"], vals, scale=scale)
        c = o.chisq_batch(d, ["q", "iangle"], vals, scale=scale, nthreads=8)
        assert np.all(np.isfinite(g))
        assert rel_err(g, c) < 1e-4


def test_chisq_batch_unphysical_is_nan(lcb):
    m = lcb.Model(GOLDEN / "test_model.dat")
    d = lcb.make_data(np.linspace(-0.2, 1.2, 50), flux=0.0, ferr=1.0, weight=1.0)
    out = m.chisq_batch(d, ["r2", "bogus"], np.array([[0.99, 1.0], [-1.0, 2.0]]), scale=False)
    assert np.isnan(out[0]) and np.isfinite(out[1])


def test_ragged_batch_and_resident_batch_vs_oracle(lcb, oracle, W):
    specs = W.batch_models(n=6, seed=5, nlat1=(20, 40), nlat2=(30, 60), ntime=(150, 300))
    models = [lcb.Model(text=s) for s, _ in specs]
    fid = lcb.Model(text=W.single_small()[0])
    datas, offs = [], [0]
    for i, (_, t) in enumerate(specs):
        f = fid.light_curve(times=t, expose=0.001, ndiv=1).flux
        datas.append(W.noisy_data(t, f, 0.001, 1, seed=100 + i))
        offs.append(offs[-1] + len(t))
    data = np.concatenate(datas)
    chi, calc, res = lcb.chisq_batch_ragged(models, data, offs, scale=False, want_calc=True)
    ochi = oracle.chisq_ragged([oracle.Model(text=s) for s, _ in specs], data, offs, scale=False, nthreads=8)
    assert rel_err(chi, ochi) < 1e-4
    for i, (s, t) in enumerate(specs):
        o = oracle.Model(text=s).light_curve(data[offs[i]:offs[i + 1]], rdata=True, nthreads=8)
        assert rel_err(calc[offs[i]:offs[i + 1]], o["calc"]) < TOL
    B = lcb.Batch(models, data, offs)
    B.run(scale=False)
    bchi, bcalc, _ = B.results(want_calc=True)
    assert np.allclose(bchi, chi, rtol=1e-12, atol=0)
    B.run(scale=False)  # graph replay
    bchi2, _, _ = B.results()
    assert np.allclose(bchi2, chi, rtol=1e-12, atol=0)
    # parameter update without re-upload of data
    q = np.array([m.q for m in models]) * 0.9
    B.set_params(["q"], q[:, None])
    B.run(scale=False)
    bchi3, _, _ = B.results()
    for i, (s, _) in enumerate(specs):
        om = oracle.Model(text=s)
        om.set("q", q[i])
        c = om.light_curve(data[offs[i]:offs[i + 1]], rdata=True, nthreads=8)["chisq"]
        assert abs(bchi3[i] - c) <= 1e-4 * abs(c)
    # several re-parameterisations in a row (a re-plan uploads only the tables that changed):
    # each equals a batch built fresh with those parameters
    rng = np.random.default_rng(7)
    names = ["q", "iangle", "r1", "t1", "t2"]
    for _ in range(3):
        vals = np.column_stack([rng.uniform(0.2, 0.9, len(models)), rng.uniform(78.0, 89.0, len(models)),
                                rng.uniform(0.008, 0.025, len(models)), rng.uniform(9000.0, 30000.0, len(models)),
                                rng.uniform(2600.0, 4800.0, len(models))])
        B.set_params(names, vals)
        B.run(scale=False)
        fresh = [lcb.Model(text=s) for s, _ in specs]
        for f, v in zip(fresh, vals):
            for k, x in zip(names, v):
                f.set_param(k, float(x))
        F = lcb.Batch(fresh, data, offs)
        F.run(scale=False)
        assert np.allclose(B.chisq(), F.chisq(), rtol=1e-12, atol=0)


@pytest.mark.parametrize("scale", [False, True])
def test_iscale_components_and_svd_scale_vs_oracle(lcb, oracle, W, scale):
    """iscale = 1: per-component fluxes (star 1, disc, rim, spot, star 2) and,
    with scale, the least-squares factor of each component (one-sided Jacobi
    SVD, restated by the oracle; no reference test pins nalgebra's result).
    Tolerances: fluxes 1e-5 relative, scale factors and chi-squared 1e-4
    relative (the fit amplifies the FP32 flux sum's rounding by the design
    matrix's conditioning)."""
    o = dict(W.SMALL)
    o.update(nlat1f=40, nlat1c=40, nlat2f=80, nlat2c=80, add_disc=1, opaque=1, rdisc1=0.02, rdisc2=0.3,
             texp_disc=-0.75, nrad=50, add_spot=1, temp_spot=12000.0, length_spot=0.05, expon_spot=0.0,
             epow_spot=2.0, nspot=40, absorb=0.5, iscale=1)
    text = W.model_text(**o)
    t = np.linspace(-0.2, 1.2, 900)
    # data: the model's own curve with different weights on its components, 1% noise
    base = oracle.Model(text=text).light_curve(lcb.make_data(t, expose=0.01, ndiv=3), scale=False)["calc"]
    rng = np.random.default_rng(5)
    flux = base * (1.0 + 0.1 * np.sin(3.0 * t)) * (1.0 + 0.01 * rng.standard_normal(t.size))
    d = lcb.make_data(t, expose=0.01, ndiv=3, flux=flux, ferr=0.01 * np.abs(flux), weight=1.0)
    d["weight"][::17] = 0.0  # some points out of the fit
    calc, res, o_ = gpu_and_oracle_lc(lcb, oracle, text, t, 0.01, 3, scale=scale, rdata=True, data=d)
    assert rel_err(calc, o_["calc"]) < TOL
    tol = 1e-4
    assert np.allclose(list(res.sfac), o_["sfac"], rtol=tol, atol=0), (list(res.sfac), o_["sfac"])
    assert res.chisq == pytest.approx(o_["chisq"], rel=tol)
    assert res.wnok == o_["wnok"]
    assert res.wdwarf == pytest.approx(o_["wdwarf"], rel=tol)
    if scale:
        assert not np.allclose(o_["sfac"], 1.0)  # the fit moved the factors


def test_time_split_light_curve_through_nccl_matches_light_curve(lcb):
    """sharded.light_curve_sharded through a one-rank NCCL group (device
    tensors in the all-gather) and without a group: the engine's own
    light_curve(scale=True), up to the order of the FP64 scaling sums."""
    import importlib
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    S = importlib.import_module("lcurve-rs_b200.sharded")
    m = lcb.Model(GOLDEN / "test_model.dat")
    t = np.linspace(-0.2, 1.2, 301)
    d = lcb.make_data(t, expose=0.001, ndiv=1, ferr=0.01, weight=1.0)
    d["flux"] = 0.02 + 0.005 * np.cos(2 * np.pi * t)
    d["weight"][::17] = 0.0
    ref = m.light_curve(data=d, scale=True)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        a = S.light_curve_sharded(m, d, scale=True, group=dist.group.WORLD)
    finally:
        dist.destroy_process_group()
    b = S.light_curve_sharded(m, d, scale=True)
    for r in (a, b):
        assert np.allclose(r.calc, ref.calc, rtol=1e-12, atol=0)
        assert np.isclose(r.chisq, ref.chisq, rtol=1e-12) and r.wnok == ref.wnok
        assert np.isclose(r.wdwarf, ref.wdwarf, rtol=1e-12) and np.allclose(r.sfac, ref.sfac, rtol=1e-12)


def test_batch_tuning_keeps_results(lcb, W):
    """lcb_batch_set_tuning: every launch-shape choice an autotuner may set
    gives the default plan's fluxes and chi-squared, up to the FP32 summation
    order of the flux sum (fluxes 1e-6 relative, ten times inside the oracle
    bound; chi-squared 1e-4, which magnifies a flux change by about flux /
    noise = 100), and lcb_batch_get_tuning reports what was set; zeros
    restore the heuristic."""
    specs = W.batch_models(n=6, seed=5, nlat1=(20, 40), nlat2=(30, 60), ntime=(150, 300))
    models = [lcb.Model(text=s) for s, _ in specs]
    fid = lcb.Model(text=W.single_small()[0])
    datas, offs = [], [0]
    for i, (_, t) in enumerate(specs):
        f = fid.light_curve(times=t, expose=0.001, ndiv=1).flux
        datas.append(W.noisy_data(t, f, 0.001, 1, seed=100 + i))
        offs.append(offs[-1] + len(t))
    data = np.concatenate(datas)
    B = lcb.Batch(models, data, offs)
    B.run(scale=True)
    chi0, calc0, _ = B.results(want_calc=True)
    heuristic = B.tuning()
    assert B.stats()["roche_elements"] > 0
    for tune in ((1, 1, 1), (16, 16, 2), (4, 3, 0), (0, 8, 1)):
        B.set_tuning(*tune)
        got = B.tuning()
        if tune[0]:
            assert got["flux_chunks"] == tune[0]
        if tune[1]:
            assert got["roche_split"] == tune[1]
        assert got["flux_blocks_per_sm"] == (min(tune[2], heuristic["flux_blocks_per_sm"]) if tune[2]
                                             else heuristic["flux_blocks_per_sm"])
        for _ in range(2):  # the captured graph, then its replay
            B.run(scale=True)
            chi, calc, _ = B.results(want_calc=True)
            assert np.allclose(calc, calc0, rtol=1e-6, atol=0), tune
            assert np.allclose(chi, chi0, rtol=1e-4, atol=0), tune
    B.set_tuning(0, 0, 0)
    assert B.tuning() == heuristic


def test_batch_split_through_nccl_matches_the_unsplit_batch(lcb, W):
    """sharded.chisq_batch_sharded (models weighed by lcb_model_work, split by
    cost, chi-squared all-gathered) through a one-rank NCCL group, with device
    tensors in the all-gather: the same chi-squared as chisq_batch_ragged."""
    import importlib
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    S = importlib.import_module("lcurve-rs_b200.sharded")
    specs = W.batch_models(n=9, seed=13, nlat1=(20, 40), nlat2=(30, 60), ntime=(100, 250))
    models = [lcb.Model(text=s) for s, _ in specs]
    offs = np.zeros(len(specs) + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(t) for _, t in specs])
    t = np.concatenate([t for _, t in specs])
    data = lcb.make_data(t, expose=0.001, ndiv=1, ferr=0.001, weight=1.0)
    data["flux"] = 0.02 + 0.004 * np.cos(2 * np.pi * t)
    ref, _, _ = lcb.chisq_batch_ragged(models, data, offs, scale=True)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        got = S.chisq_batch_sharded(models, data, offs, scale=True, group=dist.group.WORLD)
    finally:
        dist.destroy_process_group()
    assert np.all(np.isfinite(ref)) and np.allclose(got, ref, rtol=1e-12, atol=0)
    assert np.allclose(S.chisq_batch_sharded(models, data, offs, scale=True), ref, rtol=1e-12, atol=0)


def test_element_slabs_match_light_curve(lcb, W):
    """lcb_model_elements in two slabs, concatenated on the device, then
    lcb_light_curve_elements: lcb_light_curve's fluxes (the records are per
    element, the flux plan is the same); and sharded.light_curve_element_split
    through a one-rank NCCL group: Model.light_curve(scale=True)."""
    import importlib
    import socket
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    S = importlib.import_module("lcurve-rs_b200.sharded")
    text, t, expose, ndiv = W.single_large(nlat1=60, nlat2=120, ntime=600, nrad=60, nspot=40)
    m = lcb.Model(text=text)
    d = lcb.make_data(t, expose=expose, ndiv=ndiv, ferr=0.01, weight=1.0)
    d["flux"] = 0.02 + 0.004 * np.cos(2 * np.pi * t)
    ref = m.light_curve(data=d, scale=False)
    src = S.EngineElements(m)
    total = src.total()
    k = total // 3
    full = [torch.cat([x, y]) for x, y in zip(src.slab(0, k), src.slab(k, total - k))]
    calc, per = src.evaluate(full, d)
    assert np.allclose(calc, ref.calc, rtol=1e-12, atol=0)
    assert per["wdwarf"] == pytest.approx(ref.wdwarf, rel=1e-12)
    ref_s = m.light_curve(data=d, scale=True)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120), device_id=torch.device("cuda", 0))
    try:
        r = S.light_curve_element_split(m, d, scale=True, group=dist.group.WORLD)
    finally:
        dist.destroy_process_group()
    assert np.allclose(r.calc, ref_s.calc, rtol=1e-12, atol=0)
    assert r.chisq == pytest.approx(ref_s.chisq, rel=1e-12) and r.wnok == ref_s.wnok
