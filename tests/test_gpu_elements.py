"""Per-element parity of the GPU grids against the oracle: positions, normals,
areas, gravities, continuum fluxes and eclipse (ingress, egress) pairs.

The eclipse pairs must agree as sets; the FP64 Roche search on the GPU skips
line-of-sight searches only where a rigorous lower bound proves a miss, so the
intervals match the oracle's to rounding (delta_phase = 1e-7 bounds any
bisection that would take a different branch).
"""
import importlib

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def W():
    return importlib.import_module("lcurve-rs_b200.workloads")


def pair_sets(ecl):
    out = []
    for row in ecl:
        ps = sorted((row[2 * k], row[2 * k + 1]) for k in range(4) if np.isfinite(row[2 * k]) and row[2 * k] <= 2.0)
        out.append(ps)
    return out


def compare_grid(g, o, which, delta=1e-7):
    assert g["posn"].shape == o["posn"].shape, which
    n = g["posn"].shape[0]
    if n == 0:
        return 0
    assert np.max(np.abs(g["posn"] - o["posn"])) < 1e-12, which
    assert np.max(np.abs(g["dirn"] - o["dirn"])) < 1e-12, which
    assert np.allclose(g["area"], o["area"], rtol=2e-7, atol=0), which
    assert np.allclose(g["gravity"], o["gravity"], rtol=2e-7, atol=0), which
    assert np.allclose(g["flux"], o["flux"], rtol=1e-6, atol=0), which
    gs = pair_sets(g["ecl"])
    os_ = [sorted((row[2 * k], row[2 * k + 1]) for k in range(int(c))) for row, c in zip(o["ecl"], o["necl"])]
    off = 0
    for i in range(n):
        assert len(gs[i]) == len(os_[i]), (which, i, gs[i], os_[i])
        for (a, b), (c, d) in zip(gs[i], os_[i]):
            err = max(abs(a - c), abs(b - d))
            assert err <= 2 * delta, (which, i, gs[i], os_[i])
            off += err > 1e-12
    assert off <= max(1, n // 100), (which, off, n)
    return n


@pytest.mark.parametrize("case", ["golden", "disc_spot", "lensing_spots"])
def test_grids_match_oracle(lcb, oracle, W, case):
    if case == "golden":
        text = (GOLDEN / "test_model.dat").read_text()
    elif case == "disc_spot":
        text = W.single_large(nlat1=30, nlat2=60, ntime=10, nrad=40, nspot=30)[0]
    else:
        text = W.single_huge(nlat1=30, nlat2=60, ntime=10, nrad=40)[0]
    m = lcb.Model(text=text)
    og = oracle.Model(text=text).grids()
    total = 0
    for which in ("star1f", "star2f", "star1c", "star2c", "disc", "edge", "spot"):
        total += compare_grid(m.grid(which), og[which], which)
    assert total > 0


def test_roche_search_counts_and_skips(lcb, oracle, W):
    specs = W.batch_models(n=4, seed=9, nlat1=(30, 40), nlat2=(30, 40), ntime=(50, 60))
    models = [lcb.Model(text=s) for s, _ in specs]
    offs = np.cumsum([0] + [len(t) for _, t in specs])
    data = lcb.make_data(np.concatenate([t for _, t in specs]), flux=1.0, ferr=0.01)
    B = lcb.Batch(models, data, offs)
    B.run()
    c = B.search_counts()
    assert c["searches"] > 0 and c["proven_misses"] > 0
    assert c["proven_misses"] <= c["searches"]
    # the device makes exactly the reference path's line-of-sight searches (a proven
    # miss replaces a search's evaluations, not its decision)
    oracle.counters_reset()
    for (text, t), lo, hi in zip(specs, offs[:-1], offs[1:]):
        oracle.Model(text=text).light_curve(data[lo:hi], nthreads=1)
    ref = oracle.counters()["fblink"]
    assert c["searches"] == ref, (c, ref)


def test_diag_identities_on_gpu_grids(lcb, oracle, W):
    """crates/lcurve/examples/diag.rs:31-55 on the GPU's grids: the spherical
    star's area and flux sums approach 4 pi r1^2 and planck(550, t1) 4 pi r1^2
    at second order, and equal the oracle's sums to f32 rounding; the Roche
    secondary's area converges at second order too."""
    import math
    from test_oracle_golden import _sphere_text, sphere_sums
    r1, t1 = 0.015, 15000.0
    exact = 4.0 * math.pi * r1 * r1
    bb = oracle.lib().orc_planck(550.0, t1)
    errs = []
    for nlat in (20, 50, 100, 200):
        text = _sphere_text(nlat, W)
        area, flux = sphere_sums(lcb.Model(text=text).grid("star1f"))
        oarea, oflux = sphere_sums(oracle.Model(text=text).grids()["star1f"])
        assert area == pytest.approx(oarea, rel=1e-6) and flux == pytest.approx(oflux, rel=1e-6)
        assert abs(flux / (bb * area) - 1.0) < 1e-6
        errs.append(abs(area / exact - 1.0))
        assert errs[-1] < 0.1 * (math.pi / nlat) ** 2
    assert errs == sorted(errs, reverse=True) and 2.5 < errs[1] / errs[2] < 6.0
    areas = []
    for nlat in (50, 100, 200):
        text = W.model_text(nlat1f=10, nlat1c=10, nlat2f=nlat, nlat2c=nlat, eclipse1=0, eclipse2=0)
        areas.append(sphere_sums(lcb.Model(text=text).grid("star2f"))[0])
    d1, d2 = areas[1] - areas[0], areas[2] - areas[1]
    assert 2.5 < d1 / d2 < 6.0, areas
