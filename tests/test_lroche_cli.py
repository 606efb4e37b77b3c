"""The lroche front end (src/main.rs of the reference): arguments, errors and
output lines.  GPU tests run it on the reference's golden model and compare
with the golden light curve (tests/golden/test_lc.dat, C++ lroche output) and
the oracle."""
import pathlib
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rust_disp, rust_e

LROCHE = ROOT / "lcurve-rs_b200" / "lroche"


def run(*args, **kw):
    return subprocess.run([str(LROCHE), *map(str, args)], capture_output=True, text=True, timeout=300, **kw)


def test_usage_and_argument_errors():
    assert LROCHE.exists(), "build with `make -C lcurve-rs_b200`"
    r = run("--help")
    assert r.returncode == 0 and "--ntime" in r.stderr
    r = run(GOLDEN / "test_model.dat")  # one positional argument
    assert r.returncode == 2
    r = run("/nonexistent/model.dat", "none")
    assert r.returncode != 0 and "cannot open" in r.stderr


@pytest.mark.gpu
def test_golden_model_light_curve_file(tmp_path):
    out = tmp_path / "lc.dat"
    r = run(GOLDEN / "test_model.dat", "none", "--time1", -0.2, "--time2", 1.2, "--ntime", 500, "-o", out)
    assert r.returncode == 0, r.stderr
    assert "White dwarf's contribution = " in r.stdout and f"Written data to {out}" in r.stdout
    g, rf = np.loadtxt(out), np.loadtxt(GOLDEN / "test_lc.dat")
    assert g.shape == rf.shape
    # the same times (printed with 16 significant digits, as main.rs does, so to 1e-14), columns
    # and, within 1e-5, fluxes
    assert np.allclose(g[:, 0], rf[:, 0], rtol=1e-14, atol=1e-15)
    assert np.array_equal(g[:, [1, 3, 4, 5]], rf[:, [1, 3, 4, 5]])
    assert np.max(np.abs(g[:, 2] - rf[:, 2]) / np.abs(rf[:, 2])) < 1e-5
    # each line formatted as main.rs:108-116 writes it: "{:20.15e} {} {:17.10e} {} {} {}"
    for line, row in zip(out.read_text().splitlines(), g):
        want = " ".join([rust_e(row[0], 15).rjust(20), rust_disp(row[1]), rust_e(row[2], 10).rjust(17),
                         rust_disp(row[3]), rust_disp(row[4]), str(int(row[5]))])
        assert line == want, (line, want)


@pytest.mark.gpu
def test_data_file_chi_squared_matches_oracle(tmp_path, oracle):
    rng = np.random.default_rng(2)
    ref = np.loadtxt(GOLDEN / "test_lc.dat")
    data = tmp_path / "data.dat"
    flux = ref[:, 2] * 1.7 * (1.0 + 0.01 * rng.standard_normal(len(ref)))
    np.savetxt(data, np.column_stack([ref[:, 0], ref[:, 1], flux, 0.01 * flux, np.ones(len(ref)),
                                      np.ones(len(ref), int)]), fmt=["%.17g", "%.6g", "%.10g", "%.10g", "%d", "%d"])
    r = run(GOLDEN / "test_model.dat", data, "--scale")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.split("\n")
    chi = float(lines[0].split("=")[1].split(",")[0])
    sfac = float(lines[1].split("=")[1])
    from oracle import oracle as O
    o = O.Model(GOLDEN / "test_model.dat").light_curve(_read(data), scale=True, rdata=True, nthreads=8)
    assert chi == pytest.approx(o["chisq"], rel=1e-4)
    assert sfac == pytest.approx(o["sfac"][0], rel=1e-5)


def _read(path):
    from oracle import oracle as O
    a = np.loadtxt(path)
    return O.make_data(a[:, 0], expose=a[:, 1], ndiv=a[:, 5].astype(int), flux=a[:, 2], ferr=a[:, 3],
                       weight=a[:, 4])
