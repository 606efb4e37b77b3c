"""A seeded sweep of 100 models across the path's physical options (the kinds
the reference's own 100-model regression covers, test_data/
run_regression100.py: basic Roche secondaries, spherical secondaries, eclipse
flags, gravity darkening, limb-darkening laws, discs, bright spots, discs with
spots, edge cases), each light curve at 50 times in [-0.2, 1.2] on the GPU
against the oracle.  The reference's threshold there is max relative error
1e-5 (run_regression100.py:33), the same as here.  Where the oracle's light
curve is NaN (a ginterp ratio of two zero sums when the primary is eclipsed at
phase1, orchestration.rs:93-131) the GPU's must be NaN at the same points,
and where it is exactly 0 (t2 < 0 with the primary eclipsed) so must the GPU's.
"""
import importlib
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_model_sweep_vs_oracle(lcb, oracle):
    W = importlib.import_module("lcurve-rs_b200.workloads")
    sweep = W.model_sweep(n=100, seed=42)
    t = np.linspace(-0.2, 1.2, 50)
    d = lcb.make_data(t, expose=0.001, ndiv=1, ferr=1.0, weight=0.0)

    def ref(text):
        return oracle.Model(text=text).light_curve(d, nthreads=1)["calc"]

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        refs = list(ex.map(ref, [text for _, text in sweep]))
    finite_models, worst = 0, {}
    for (kind, text), o in zip(sweep, refs):
        g = lcb.Model(text=text).light_curve(times=t, expose=0.001, ndiv=1).flux
        assert np.array_equal(np.isnan(g), np.isnan(o)), kind
        # exact zeros (both stars dark or hidden: t2 < 0 and the primary eclipsed) must be zeros
        assert np.array_equal(g[o == 0.0], o[o == 0.0]), kind
        ok = np.isfinite(o) & (o != 0.0)
        if ok.any():
            err = float(np.max(np.abs(g[ok] - o[ok]) / np.abs(o[ok])))
            worst[kind] = max(worst.get(kind, 0.0), err)
            assert err < TOL, (kind, err)
        finite_models += bool(ok.all())
    print("max rel err per kind:", {k: f"{v:.1e}" for k, v in worst.items()})
    assert finite_models >= 80
    assert set(worst) == set(W.SWEEP_KINDS)
