"""Pins the CPU oracle against the reference's golden vectors and known answers.

Golden: test_data/test_lc.dat of the reference, 500 fluxes written by the C++
lroche for test_data/test_model.dat at times -0.2..1.2, expose 0.001, ndiv 1;
the reference's own bound is max relative error < 1e-6 (tests/regression.rs:84-88).
"""
import math

import numpy as np
import pytest

from conftest import GOLDEN


def golden_data(O):
    t = -0.2 + 1.4 * np.arange(500) / 499
    return O.make_data(t, expose=0.001, ndiv=1, flux=0.0, ferr=0.0, weight=1.0)


def test_oracle_matches_cpp_golden(oracle, test_model_path):
    m = oracle.Model(test_model_path)
    r = m.light_curve(golden_data(oracle), scale=False, rdata=False, nthreads=4)
    g = np.loadtxt(GOLDEN / "test_lc.dat")
    assert np.array_equal(golden_data(oracle)["time"], g[:, 0])
    rel = np.abs(r["calc"] - g[:, 2]) / np.abs(g[:, 2])
    # The golden carries 10 significant digits; observed max ~1.4e-10.
    assert rel.max() < 1e-9, rel.max()


def test_oracle_threading_is_bitwise_stable(oracle, test_model_path):
    m = oracle.Model(test_model_path)
    a = m.light_curve(golden_data(oracle), nthreads=1)["calc"]
    b = m.light_curve(golden_data(oracle), nthreads=8)["calc"]
    assert np.array_equal(a, b)


def test_lagrange_known_answers(oracle):
    L = oracle.lib()
    # lagrange.rs:148-152, 172-184
    assert abs(L.orc_xl1(1.0) - 0.5) < 1e-10
    assert 0.0 < L.orc_xl1(0.1) < 1.0
    assert abs(L.orc_xl1(0.5) - L.orc_xl11(0.5, 1.0)) < 1e-10
    assert abs(L.orc_xl1(0.5) - L.orc_xl12(0.5, 1.0)) < 1e-10
    assert math.isnan(L.orc_xl1(-1.0))


def test_planck_known_answers(oracle):
    L = oracle.lib()
    # planck.rs:49-75
    assert L.orc_planck(500.0, 10000.0) > L.orc_planck(500.0, 5000.0) > 0.0
    assert L.orc_planck(100.0, 100.0) >= 0.0
    assert L.orc_dlpdlt(500.0, 10000.0) > 0.0 and L.orc_dlpdlt(500.0, 3000.0) > 0.0


def test_numface_table(oracle):
    # Element counts per latitude resolution (grid.rs:8-46).
    L = oracle.lib()
    expect = {20: 540, 40: 2058, 50: 3202, 100: 12724, 200: 50872, 400: 203560}
    for nlat, n in expect.items():
        assert L.orc_numface(nlat) == n


def test_stream_spot_position(oracle):
    # The stream reaches the requested radius (stream.rs:82-145) from just inside L1.
    import ctypes as C
    out = (C.c_double * 3)()
    oracle.lib().orc_stream_spot(0.5, 0.3, out)
    r = math.sqrt(out[0] ** 2 + out[1] ** 2 + out[2] ** 2)
    assert abs(r - 0.3) < 1e-9
    assert out[2] == 0.0
    # a radius the stream never reaches is the reference's error (stream.rs:139-141): NaN here
    oracle.lib().orc_stream_spot(0.08, 0.12, out)
    assert all(math.isnan(x) for x in out)


def test_parse_errors(oracle, tmp_path):
    text = (GOLDEN / "test_model.dat").read_text()
    with pytest.raises(oracle.OracleError):
        oracle.Model(text=text + "\nbogus_param = 1\n")
    with pytest.raises(oracle.OracleError):
        oracle.Model(text=text.replace("limb1                = Poly", "limb1 = Quadratic"))
    with pytest.raises(oracle.OracleError):
        oracle.Model(text=text + "\nstsp11_long = 10 1 1 0\n")
    m = oracle.Model(text=text)
    assert m.get("q") == 0.5 and m.get("pdot") == 0.0


def test_chisq_batch_matches_sequential(oracle, test_model_path):
    # tests/chisq_batch.rs:50-89 (batch == sequential to 1e-10)
    m = oracle.Model(test_model_path)
    t = -0.2 + 1.4 * np.arange(100) / 99
    d = oracle.make_data(t, expose=0.001, ndiv=1, flux=0.0, ferr=1.0, weight=1.0)
    q0 = m.get("q")
    offs = [-0.02, 0.0, 0.02]
    vals = np.array([[q0 + dq, m.get("iangle")] for dq in offs])
    batch = m.chisq_batch(d, ["q", "iangle"], vals, scale=False, nthreads=3)
    for i, dq in enumerate(offs):
        mm = m.clone()
        mm.set("q", q0 + dq)
        seq = mm.light_curve(d, scale=False, rdata=True)["chisq"]
        assert abs(batch[i] - seq) < 1e-10 * max(abs(seq), 1.0)


def test_chisq_batch_unphysical_is_nan(oracle, test_model_path):
    # tests/chisq_batch.rs:92-109
    m = oracle.Model(test_model_path)
    t = -0.2 + 1.4 * np.arange(50) / 49
    d = oracle.make_data(t, flux=0.0, ferr=1.0, weight=1.0)
    out = m.chisq_batch(d, ["r2"], np.array([[0.99]]))
    assert np.isnan(out[0])


def _svd_lstsq(flux, ferr, weight, fcomp):
    """svd_scale restated through LAPACK's SVD: rows with weight > 0 scaled by
    sqrt(weight) / ferr, x = V S^+ U^T b with singular values below 1e-12
    (absolute, as nalgebra's SVD::solve(b, 1e-12)) treated as zero."""
    use = weight > 0
    ncol = fcomp.shape[1]
    if use.sum() < ncol or use.sum() == 0:
        return np.ones(ncol)
    w = np.sqrt(weight[use]) / ferr[use]
    a, b = fcomp[use] * w[:, None], flux[use] * w
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    keep = s >= 1e-12
    return vt.T[:, keep] @ ((u.T[keep] @ b) / s[keep])


def test_svd_scale_restatement_against_lapack(oracle):
    """The oracle's one-sided Jacobi least squares (svd_scale, the iscale = 1
    path; orchestration.rs:405-436) against the same problem solved through
    LAPACK: well-conditioned, an all-zero component (singular value 0: its
    factor is 0), two identical components (the minimum-norm split) and too
    few weighted rows (all ones)."""
    import ctypes as C
    L = oracle.lib()
    rng = np.random.default_rng(9)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    cases = []
    for ncol in (4, 5):
        n = 300
        fcomp = np.abs(rng.normal(1.0, 0.5, (n, ncol))) * np.array([1.0, 0.3, 0.05, 0.02, 0.5])[:ncol]
        truth = rng.uniform(0.5, 2.0, ncol)
        ferr = rng.uniform(0.005, 0.02, n)
        flux = fcomp @ truth + rng.normal(0.0, 1.0, n) * ferr
        weight = np.where(rng.random(n) < 0.1, 0.0, rng.uniform(0.5, 2.0, n))
        cases.append((flux, ferr, weight, fcomp, 1e-10))
        zero = fcomp.copy()
        zero[:, 2] = 0.0
        cases.append((zero @ truth, ferr, weight, zero, 1e-10))
        twin = fcomp.copy()
        twin[:, 1] = twin[:, 0]
        cases.append((twin @ truth, ferr, weight, twin, 1e-8))
    few = np.ones((3, 5))
    cases.append((np.ones(3), np.ones(3), np.ones(3), few, 0.0))
    for flux, ferr, weight, fcomp, tol in cases:
        out = np.zeros(fcomp.shape[1])
        fc = np.ascontiguousarray(fcomp)
        L.orc_svd_scale(dp(np.ascontiguousarray(flux)), dp(np.ascontiguousarray(ferr)),
                        dp(np.ascontiguousarray(weight)), fcomp.shape[0], dp(fc), fcomp.shape[1], dp(out))
        ref = _svd_lstsq(flux, ferr, weight, fcomp)
        assert np.allclose(out, ref, rtol=tol, atol=tol * np.max(np.abs(ref))), (out, ref)


def test_roche_unit_known_answers(oracle):
    """The reference roche crate's own unit tests, on the oracle's restatements:
    set_earth at i = 90 (misc.rs:58-69), the potential's sign (potential.rs:
    133-142), zero gradient at L1 (potential.rs:145-152), strinit just inside
    L1 (stream.rs:282-289) and the Jacobi constant over one gsint step
    (stream.rs:292-309; jacobi from misc.rs:21-28), ref_sphere and face on the
    primary (surface.rs:128-146)."""
    import ctypes as C
    L = oracle.lib()
    v3 = lambda: (C.c_double * 3)()  # noqa: E731
    e = v3()
    L.orc_set_earth(90.0, 0.0, e)
    assert abs(e[0] - 1.0) < 1e-10 and abs(e[1]) < 1e-10 and abs(e[2]) < 1e-10
    L.orc_set_earth(90.0, 0.25, e)
    assert abs(e[0]) < 1e-10 and abs(e[1] + 1.0) < 1e-10
    assert math.isfinite(L.orc_rpot(1.0, 0.5, 0.0, 0.0))
    assert L.orc_rpot(1.0, 0.1, 0.0, 0.0) < 0.0
    g = v3()
    L.orc_drpot1(1.0, 1.0, L.orc_xl1(1.0), 0.0, 0.0, g)
    assert abs(g[0]) < 1e-10 and abs(g[1]) < 1e-15 and abs(g[2]) < 1e-15
    r, v = v3(), v3()
    L.orc_strinit(1.0, r, v)
    assert 0.0 < r[0] < 0.5 and abs(r[1]) < 0.01 and r[2] == 0.0 and v[0] < 0.0

    def jacobi(q, s):
        f1 = 1.0 / (1.0 + q)
        f2 = f1 * q
        yzsq = s[1] ** 2 + s[2] ** 2
        return ((s[3] ** 2 + s[4] ** 2 + s[5] ** 2 - s[1] ** 2 - (s[0] - f2) ** 2) / 2.0
                - f1 / math.sqrt(s[0] ** 2 + yzsq) - f2 / math.sqrt((s[0] - 1.0) ** 2 + yzsq))

    s0, s1 = (C.c_double * 6)(), (C.c_double * 6)()
    L.orc_gsint_step(0.5, 0.01, 1e-10, s0, s1)
    assert list(s0) != list(s1)
    assert abs(jacobi(0.5, s0) - jacobi(0.5, s1)) < 1e-8
    # ref_sphere and face (surface.rs:128-146)
    rp = (C.c_double * 2)()
    L.orc_ref_sphere(1.0, 1, 1.0, 1.0, rp)
    assert rp[0] > 0.0 and rp[1] < 0.0
    p, d, rg = v3(), v3(), (C.c_double * 2)()
    L.orc_face(0.5, 0, 1.0, 0.9, (C.c_double * 3)(0.0, 1.0, 0.0), 1e-6, p, d, rg)
    assert rg[0] > 0.0 and rg[1] > 0.0 and p[1] > 0.0


def test_numerical_known_answers(oracle):
    """The subs crate's numerical unit tests on the oracle's restatements:
    dbrent finds the minimum of (x - 3)^2 + 1 from (0, 2, 6) (dbrent.rs:
    172-181); one Bulirsch-Stoer step of dy/dx = y matches e^x at the x it
    reached (bsstep.rs:570-597)."""
    import ctypes as C
    L = oracle.lib()
    fx = (C.c_double * 2)()
    assert L.orc_dbrent_quadratic(fx) in (0, 1)
    assert abs(fx[1] - 3.0) < 1e-9 and abs(fx[0] - 1.0) < 1e-9
    yx = (C.c_double * 2)()
    L.orc_bsstep_exp(yx)
    assert yx[1] > 0.0 and abs(yx[0] - math.exp(yx[1])) / math.exp(yx[1]) < 1e-8


# ---- crates/lcurve/examples/diag.rs:31-55: grid and continuum identities ----
def _sphere_text(nlat, W):
    # the golden model's spherical white dwarf (roche1 = 0, r1 = 0.015); absorb = 0: no
    # irradiation, so each element's flux is its area times planck(wavelength, t1); eclipses off
    # (they change no area or flux)
    return W.model_text(nlat1f=nlat, nlat1c=nlat, nlat2f=10, nlat2c=10, absorb=0.0, eclipse1=0, eclipse2=0)


def sphere_sums(g):
    return float(np.sum(g["area"].astype(np.float64))), float(np.sum(g["flux"].astype(np.float64)))


def test_diag_sphere_area_and_flux_identities(oracle):
    """Sum of star 1's element areas -> 4 pi r1^2 and sum of fluxes -> planck(550 nm, t1)
    4 pi r1^2 (diag.rs:34-55); the latitude bands are a midpoint rule in theta, so the
    relative error is about (pi / nlat)^2 / 24 and falls as 1 / nlat^2."""
    import importlib
    W = importlib.import_module("lcurve-rs_b200.workloads")
    r1, t1 = 0.015, 15000.0
    exact = 4.0 * math.pi * r1 * r1
    bb = oracle.lib().orc_planck(550.0, t1)
    errs = []
    for nlat in (20, 50, 100, 200):
        area, flux = sphere_sums(oracle.Model(text=_sphere_text(nlat, W)).grids()["star1f"])
        e = area / exact - 1.0
        assert abs(e) < 0.1 * (math.pi / nlat) ** 2, (nlat, e)
        assert abs(flux / (bb * area) - 1.0) < 1e-6  # per element f32 rounding only
        assert abs(flux / (bb * exact) - 1.0) < 0.1 * (math.pi / nlat) ** 2
        errs.append(abs(e))
    assert errs == sorted(errs, reverse=True)
    assert 2.5 < errs[1] / errs[2] < 6.0  # second order: halving the spacing quarters the error


def test_diag_roche_star_area_converges(oracle):
    """The Roche-lobe-filling secondary's area at nlat 50/100/200 converges at
    second order (successive differences shrink about four-fold)."""
    import importlib
    W = importlib.import_module("lcurve-rs_b200.workloads")
    areas = []
    for nlat in (50, 100, 200):
        text = W.model_text(nlat1f=10, nlat1c=10, nlat2f=nlat, nlat2c=nlat, eclipse1=0, eclipse2=0)
        areas.append(sphere_sums(oracle.Model(text=text).grids()["star2f"])[0])
    d1, d2 = areas[1] - areas[0], areas[2] - areas[1]
    assert abs(d2) < abs(d1)
    assert 2.5 < d1 / d2 < 6.0, (areas, d1, d2)
