"""Parity at the full sizes of the large single-model workloads.

single_large (nlat 200/400, opaque disc nrad 200, rim, bright spot,
irradiation, 10,000 times x 5 sub-divisions): every flux of the GPU light
curve against the oracle's, max relative error 1e-5 (the reference's own
GPU-vs-CPU bound is 1e-3, crates/lcurve-cuda/tests/gpu_correctness.rs:109-114;
its CPU regression bound 1e-6, tests/regression.rs:84-88), and every element
of every grid (positions, normals, areas, gravities, fluxes, eclipse pairs).

single_huge (nlat 400/800, disc nrad 1000 with rim, two star spots on star 2,
lensing; ~5.1 M elements): every element of every grid against the oracle's,
and the light curve at 1,000 of its 100,000 times (every 100th, all 11
sub-divisions: 5.6e10 oracle element-evaluations) against the oracle's
light curve on its own grids.

The oracle builds these grids with its eclipse intervals computed on all host
threads (orc_set_grid_threads): the same per-element function as the
reference's serial add_faces, only faster.
"""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5
THREADS = os.cpu_count() or 1
GRIDS = ("star1f", "star2f", "star1c", "star2c", "disc", "edge", "spot")


@pytest.fixture(scope="module")
def W():
    return importlib.import_module("lcurve-rs_b200.workloads")


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def sorted_pairs(ing, eg):
    """(n, 4) ingress and egress arrays with empty slots = +inf, each row's pairs
    sorted by (ingress, egress)."""
    n = ing.shape[0]
    row = np.repeat(np.arange(n), 4)
    order = np.lexsort((eg.ravel(), ing.ravel(), row))
    return ing.ravel()[order].reshape(n, 4), eg.ravel()[order].reshape(n, 4)


def compare_grid(g, o, which, delta=1e-7):
    """Every element of one grid: positions and normals within 1e-12, area and
    gravity within f32 rounding, continuum flux within 1e-6, the same number
    of eclipse pairs with ingress and egress within 2 delta_phase, and at
    most 1% of the elements off by more than 1e-12 (a bisection that took the
    other branch within delta_phase)."""
    n = g["posn"].shape[0]
    assert n == o["posn"].shape[0], which
    if n == 0:
        return 0
    assert np.max(np.abs(g["posn"] - o["posn"])) < 1e-12, which
    assert np.max(np.abs(g["dirn"] - o["dirn"])) < 1e-12, which
    assert np.allclose(g["area"], o["area"], rtol=2e-7, atol=0), which
    assert np.allclose(g["gravity"], o["gravity"], rtol=2e-7, atol=0), which
    assert np.allclose(g["flux"], o["flux"], rtol=1e-6, atol=0), which
    gi, ge = g["ecl"][:, 0::2].copy(), g["ecl"][:, 1::2].copy()
    empty = ~(gi <= 2.0)  # unused GPU slots are (+inf, -inf)
    gi[empty], ge[empty] = np.inf, np.inf
    oi, oe = o["ecl"][:, 0::2].copy(), o["ecl"][:, 1::2].copy()
    unused = np.arange(4)[None, :] >= o["necl"][:, None]
    oi[unused], oe[unused] = np.inf, np.inf
    gi, ge = sorted_pairs(gi, ge)
    oi, oe = sorted_pairs(oi, oe)
    assert np.array_equal(np.isinf(gi), np.isinf(oi)), which  # same number of pairs per element
    used = ~np.isinf(oi)
    err = np.zeros_like(oi)
    err[used] = np.maximum(np.abs(gi[used] - oi[used]), np.abs(ge[used] - oe[used]))
    assert err.max() <= 2 * delta, which
    off = int(np.count_nonzero((err > 1e-12).any(axis=1)))
    assert off <= max(1, n // 100), (which, off, n)
    return n


def check_scalars(res, o):
    assert abs(res.wdwarf - o["wdwarf"]) <= 1e-7 * abs(o["wdwarf"])
    assert res.logg1 == pytest.approx(o["logg1"], rel=1e-12)
    assert res.logg2 == pytest.approx(o["logg2"], rel=1e-12)
    assert res.rv1 == pytest.approx(o["rv1"], rel=1e-12)
    assert res.rv2 == pytest.approx(o["rv2"], rel=1e-12)


def test_single_large_full_size(lcb, oracle, W):
    text, t, expose, ndiv = W.single_large()
    m = lcb.Model(text=text)
    r = m.light_curve(times=t, expose=expose, ndiv=ndiv)
    G = oracle.Model(text=text).built_grids(threads=THREADS)
    o = G.light_curve(oracle.make_data(t, expose=expose, ndiv=ndiv), nthreads=THREADS)
    err = rel_err(r.flux, o["calc"])
    print(f"single_large full size: {len(t)} times x {ndiv}, max rel err {err:.2e}")
    assert err < TOL
    check_scalars(r, o)
    total = sum(compare_grid(m.grid(w), G.fetch(w), w) for w in GRIDS)
    assert total > 400_000


def test_single_huge_full_grids_and_thinned_times(lcb, oracle, W):
    text, t, expose, ndiv = W.single_huge()
    m = lcb.Model(text=text)
    G = oracle.Model(text=text).built_grids(threads=THREADS)
    total = 0
    for w in GRIDS:
        total += compare_grid(m.grid(w), G.fetch(w), w)
    assert total > 5_000_000
    ts = t[::100]
    r = m.light_curve(times=ts, expose=expose, ndiv=ndiv)
    o = G.light_curve(oracle.make_data(ts, expose=expose, ndiv=ndiv), nthreads=THREADS)
    err = rel_err(r.flux, o["calc"])
    print(f"single_huge full grids ({total} elements), {len(ts)} times x {ndiv}: max rel err {err:.2e}")
    assert err < TOL
    check_scalars(r, o)
