"""lcb_light_curve_noalloc against lcb_light_curve, through the C ABI.

lcb_light_curve_noalloc serves callers that cannot call cudaMalloc — a
process whose device memory already belongs to another framework's pool
allocator, a plugin host that forbids allocation in its callbacks, a loop that
cannot take the synchronisation an allocation may bring.  It keeps all device
scratch in one fixed arena that every call on a device shares, so these tests
run it several times in a row, on models of different sizes, and check each
result against the allocating entry point.  Tolerance: max relative error
1e-5, the one the other GPU parity tests use.

This file is named to be collected last: it must pass alone in a fresh
process and after every other test.
"""
import ctypes as C
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
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _call(lcb, entry, model, data, scale):
    calc = np.zeros(data.shape[0])
    res = lcb.Result()
    fn = getattr(lcb._capi.load(), entry)
    rc = fn(lcb._ctx(), model._h, data.ctypes.data, data.shape[0], int(scale), 0, lcb._capi.dptr(calc),
            C.byref(res))
    return rc, calc, res


def _cases(lcb, W):
    """(model, data, scale) triples of different grid and data sizes."""
    a = lcb.Model(GOLDEN / "test_model.dat")
    da = lcb.make_data(np.linspace(-0.2, 1.2, 500), expose=0.001, ndiv=1, ferr=1.0, weight=1.0)
    text, t, expose, ndiv = W.single_large(nlat1=40, nlat2=80, ntime=1500, nrad=50, nspot=40)
    b = lcb.Model(text=text)
    db = lcb.make_data(t, expose=expose, ndiv=ndiv, ferr=0.01, weight=1.0)
    db["flux"] = 1.0 + 0.1 * np.sin(7.0 * t)
    return [(a, da, False), (b, db, True), (a, da, False)]


def _assert_same(res, calc, ref_res, ref_calc, scaled):
    assert rel_err(calc, ref_calc) < TOL
    assert abs(res.wdwarf - ref_res.wdwarf) <= TOL * abs(ref_res.wdwarf)
    assert res.logg1 == pytest.approx(ref_res.logg1, rel=TOL)
    assert res.logg2 == pytest.approx(ref_res.logg2, rel=TOL)
    if scaled:
        assert res.chisq == pytest.approx(ref_res.chisq, rel=TOL)
        assert np.allclose(list(res.sfac), list(ref_res.sfac), rtol=TOL, atol=0)


def test_noalloc_matches_light_curve_on_calls_in_a_row(lcb, W):
    cases = _cases(lcb, W)
    refs = []
    for m, d, scale in cases:
        rc, calc, res = _call(lcb, "lcb_light_curve", m, d, scale)
        lcb._capi.check(rc)
        refs.append((calc, res))
    # consecutive no-allocation calls: each one reuses the arena the previous one left behind
    for (m, d, scale), (ref_calc, ref_res) in zip(cases, refs):
        rc, calc, res = _call(lcb, "lcb_light_curve_noalloc", m, d, scale)
        lcb._capi.check(rc)
        _assert_same(res, calc, ref_res, ref_calc, scale)


def test_noalloc_rejects_a_model_beyond_the_arena(lcb, W):
    big = lcb.Model(text=W.model_text(nlat1f=400, nlat2f=1500))
    d = lcb.make_data(np.linspace(0.0, 1.0, 64), expose=0.001, ndiv=1, ferr=1.0, weight=1.0)
    rc, _, _ = _call(lcb, "lcb_light_curve_noalloc", big, d, False)
    assert lcb._capi.ERR_NAMES.get(rc) == "LCB_ERR_INVALID"
    msg = lcb._capi.load().lcb_last_error().decode()
    assert "bytes of device scratch" in msg and str(64 * 1024 * 1024) in msg
    # the rejected call did no device work; the next call still matches
    m, da, _ = _cases(lcb, W)[0]
    _, ref_calc, ref_res = _call(lcb, "lcb_light_curve", m, da, False)
    rc, calc, res = _call(lcb, "lcb_light_curve_noalloc", m, da, False)
    lcb._capi.check(rc)
    _assert_same(res, calc, ref_res, ref_calc, False)


def test_noalloc_allocates_no_device_memory(lcb, W):
    import torch
    m, d, scale = _cases(lcb, W)[1]
    rc, ref_calc, ref_res = _call(lcb, "lcb_light_curve", m, d, scale)
    lcb._capi.check(rc)
    lcb._capi.check(_call(lcb, "lcb_light_curve_noalloc", m, d, scale)[0])  # warm: every kernel launched once
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, calc, res = _call(lcb, "lcb_light_curve_noalloc", m, d, scale)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    lcb._capi.check(rc)
    assert free1 == free0
    _assert_same(res, calc, ref_res, ref_calc, scale)


def test_noalloc_calls_from_two_threads(lcb, W):
    """Two host threads, each with its own context on the same device, call the
    entry point at once: the calls share the arena, so the library must run
    them one at a time, and every result must still match."""
    import threading

    L = lcb._capi.load()
    cases = _cases(lcb, W)[:2]
    refs = []
    for m, d, scale in cases:
        rc, calc, res = _call(lcb, "lcb_light_curve", m, d, scale)
        lcb._capi.check(rc)
        refs.append((calc, res))
    dev = int(str(lcb.get_device()).split(":")[-1]) if ":" in str(lcb.get_device()) else 0
    ctxs = []
    for _ in range(2):
        h = C.c_void_p()
        lcb._capi.check(L.lcb_ctx_create(dev, C.byref(h)))
        ctxs.append(h)
    errors = []

    def worker(k):
        m, d, scale = cases[k]
        ref_calc, ref_res = refs[k]
        try:
            for _ in range(4):
                calc = np.zeros(d.shape[0])
                res = lcb.Result()
                rc = L.lcb_light_curve_noalloc(ctxs[k], m._h, d.ctypes.data, d.shape[0], int(scale), 0,
                                               lcb._capi.dptr(calc), C.byref(res))
                assert rc == 0, rc
                _assert_same(res, calc, ref_res, ref_calc, scale)
        except BaseException as e:  # noqa: BLE001 (reported by the main thread)
            errors.append(e)

    try:
        threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
    finally:
        for h in ctxs:
            L.lcb_ctx_destroy(h)
    assert not errors, errors
