"""The failure contract on the GPU, driven without faulting anything.

The reference maps a model whose light curve fails to NaN in chisq_batch
(crates/lcurve/src/orchestration.rs:350-354) and returns the error from
light_curve_comp.  Here the device's own bounds play that role:

* the eclipse search's cap on one line-of-sight search (the reference's
  fblink, crates/roche/src/eclipse.rs:123-197, has none): lowered for one
  context with lcb_ctx_set_search_cap, it must turn exactly the models that
  need the Roche search into NaN (chisq entry points, resident batches) or
  LCB_ERR_DEVICE_CHECK (lcb_light_curve), and the next call with the default
  cap must be exact again;
* the bounded mbarrier wait of the flux kernel's copy pipeline: a probe
  waits on a barrier nothing completes (no copy in flight, no arrival); the
  wait must give up after its limit, report LCB_ERR_DEVICE_CHECK, and leave
  the context usable.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

DEVICE_CHECK = 9


def _models(lcb):
    roche = lcb.Model(GOLDEN / "test_model.dat")  # star 2 fills its Roche lobe: star 1 needs the Roche search
    sphere = roche.copy()
    sphere.set_comp("roche2", "0")  # both stars spheres: analytic eclipses only, the cap never applies
    for k in ("nlat1c", "nlat2c"):    # one grid per star (no ginterp ratio, which is 0/0 when the
        sphere.set_comp(k, sphere.get_comp(k.replace("c", "f")))  # larger sphere hides star 1 at phase1)
    return roche, sphere


def test_search_cap_fails_the_roche_models_and_the_default_recovers(lcb):
    L, ctx = lcb._capi.load(), lcb._ctx()
    roche, sphere = _models(lcb)
    t = np.linspace(-0.2, 1.2, 200)
    good = roche.light_curve(times=t, expose=0.001, ndiv=1).flux
    base = sphere.light_curve(times=t, expose=0.001, ndiv=1).flux
    one = lcb.make_data(t, expose=0.001, ndiv=1, flux=good * 1.01, ferr=0.01 * good, weight=1.0)
    data = np.concatenate([one, one])
    offs = np.array([0, len(t), 2 * len(t)], dtype=np.int64)
    B = lcb.Batch([roche, sphere], data, offs)
    B.run(scale=False)
    ok_chi, _, _ = B.results()
    assert np.all(np.isfinite(ok_chi))
    lcb._capi.check(L.lcb_ctx_set_search_cap(ctx, 2))
    try:
        chi, _, res = lcb.chisq_batch_ragged([roche, sphere], data, offs, scale=False)
        assert np.isnan(chi[0]) and np.isnan(res[0].wdwarf)
        assert chi[1] == pytest.approx(ok_chi[1], rel=1e-12)
        with pytest.raises(lcb.LcbError) as e:
            roche.light_curve(times=t, expose=0.001, ndiv=1)
        assert e.value.code == DEVICE_CHECK and "iteration cap" in str(e.value)
        assert np.array_equal(sphere.light_curve(times=t, expose=0.001, ndiv=1).flux, base)
        B.run(scale=False)  # the resident batch's graph is captured again with the lowered cap
        bchi, _, _ = B.results()
        assert np.isnan(bchi[0]) and bchi[1] == pytest.approx(ok_chi[1], rel=1e-12)
    finally:
        lcb._capi.check(L.lcb_ctx_set_search_cap(ctx, 0))
    # restored: the results before (the per-model sums behind the ginterp scale factors are
    # FP64 atomics, so the last bits may differ from run to run)
    assert np.allclose(roche.light_curve(times=t, expose=0.001, ndiv=1).flux, good, rtol=1e-12, atol=0)
    B.run(scale=False)
    bchi, _, _ = B.results()
    assert np.allclose(bchi, ok_chi, rtol=1e-12, atol=0)
    g = np.loadtxt(GOLDEN / "test_lc.dat")
    r = lcb.Model(GOLDEN / "test_model.dat").light_curve(time1=-0.2, time2=1.2, ntime=500, expose=0.001, ndiv=1)
    assert np.max(np.abs(r.flux - g[:, 2]) / np.abs(g[:, 2])) < 1e-5


def test_bounded_wait_gives_up_and_the_context_stays_usable(lcb):
    L, ctx = lcb._capi.load(), lcb._ctx()
    limit = 200_000  # SM cycles, ~0.1 ms
    waited = C.c_int64()
    rc = L.lcb_wait_probe(ctx, limit, C.byref(waited))
    assert rc == DEVICE_CHECK
    assert "timed out" in L.lcb_last_error().decode()
    assert limit <= waited.value < 1000 * limit
    assert L.lcb_wait_probe(ctx, 0, C.byref(waited)) == 1  # a limit must be given
    g = np.loadtxt(GOLDEN / "test_lc.dat")
    r = lcb.Model(GOLDEN / "test_model.dat").light_curve(time1=-0.2, time2=1.2, ntime=500, expose=0.001, ndiv=1)
    assert np.max(np.abs(r.flux - g[:, 2]) / np.abs(g[:, 2])) < 1e-5
