"""The bright spot's gas stream on the GPU (lcb_stream.h compiled for the device,
k_stream): the stream from L1 to the spot radius (crates/roche/src/stream.rs:82-145
with the Bulirsch-Stoer step of crates/subs/src/numerical/bsstep.rs) integrated by
one GPU thread per (q, radius) pair, against the same source on the host, and a
batch with more new pairs than four per host thread (the planner then takes the
GPU path) against the oracle's light curves.

Tolerance of the end points: 1e-9 absolute.  The two runs share every operation;
only pow (in the step control) may round differently in its last bit on the two
processors, which can move a step size and hence the end point by rounding only,
far inside the stream's own 1e-10 radius tolerance and the 1e-4 chi-squared
tolerance of the batch parity tests.
"""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def W():
    return importlib.import_module("lcurve-rs_b200.workloads")


def _points(lcb, q, rad, device):
    out = np.zeros((len(q), 3))
    rc = lcb._capi.load().lcb_stream_points(lcb._ctx(), lcb._capi.dptr(np.ascontiguousarray(q)),
                                            lcb._capi.dptr(np.ascontiguousarray(rad)), len(q), int(device),
                                            lcb._capi.dptr(out))
    return rc, out


def test_stream_points_device_equal_host(lcb, oracle):
    L = oracle.lib()
    qs, rads = [], []
    for q in np.linspace(0.08, 1.0, 12):
        xl1 = L.orc_xl1(float(q))
        for frac in (0.35, 0.5, 0.65, 0.8):
            qs.append(float(q))
            rads.append(round(frac * xl1, 6))
    q, rad = np.array(qs), np.array(rads)
    rc_h, host = _points(lcb, q, rad, False)
    rc_d, dev = _points(lcb, q, rad, True)
    assert rc_h == 0 and rc_d == 0
    assert np.all(np.isfinite(dev))
    assert np.max(np.abs(dev - host)) < 1e-9, np.max(np.abs(dev - host))
    # the end point lies at the requested radius (the stream's own tolerance)
    assert np.max(np.abs(np.linalg.norm(dev, axis=1) - rad)) < 1e-8


def test_many_new_spot_pairs_take_the_gpu_path_and_match_the_oracle(lcb, oracle, W):
    n = 4 * (os.cpu_count() or 1) + 8  # more new pairs than four per host thread
    rng = np.random.default_rng(21)
    specs = []
    base = dict(W.SMALL)
    base.update(nlat1f=16, nlat1c=16, nlat2f=24, nlat2c=24, add_disc=1, opaque=0, rdisc1=0.02, rdisc2=0.3,
                nrad=10, add_spot=1, temp_spot=12000.0, length_spot=0.05, expon_spot=0.0, epow_spot=2.0,
                nspot=20)
    t = np.linspace(-0.2, 1.2, 40)
    for k in range(n):
        o = dict(base, q=float(rng.uniform(0.3, 0.7)), iangle=float(rng.uniform(78.0, 88.0)))
        specs.append(W.model_text(**o))
    data = lcb.make_data(np.tile(t, n), expose=0.01, ndiv=1, flux=0.02, ferr=0.001, weight=1.0)
    offs = np.arange(n + 1) * len(t)
    chi, _, _ = lcb.chisq_batch_ragged([lcb.Model(text=s) for s in specs], data, offs, scale=True)
    ref = oracle.chisq_ragged([oracle.Model(text=s) for s in specs], data, offs, scale=True, nthreads=8)
    assert np.all(np.isfinite(chi))
    assert np.max(np.abs(chi - ref) / np.abs(ref)) < 1e-4
