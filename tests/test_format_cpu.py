"""The lroche front end's number formatting (lcb_model.cpp: fmt_display,
fmt_lower_exp) against restatements of Rust's `{}` and `{:.Ne}` for f64, the
formats of the reference CLI's output lines (src/main.rs:108-116), on
random magnitudes, exact powers of two (asymmetric rounding intervals) and
their neighbours, subnormals and the extremes.  A small driver is compiled
from the library's host source; exact string equality.
"""
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rust_disp, rust_e

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include "lcb_model.h"
int main(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
        double v = std::strtod(argv[i], nullptr);
        std::printf("%s|%s|%s\n", lcb::fmt_display(v).c_str(), lcb::fmt_lower_exp(v, 15).c_str(),
                    lcb::fmt_lower_exp(v, 10).c_str());
    }
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("fmt")
    (d / "d.cpp").write_text(DRIVER)
    src = ROOT / "lcurve-rs_b200" / "csrc"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I/usr/local/cuda/include", f"-I{src}", str(d / "d.cpp"),
                    str(src / "lcb_model.cpp"), "-o", str(d / "d")], check=True)
    return d / "d"


def _values():
    rng = np.random.default_rng(0)
    v = list(rng.uniform(-1, 1, 2000) * 10.0 ** rng.integers(-300, 300, 2000))
    v += list(rng.uniform(0, 2, 500))  # the magnitudes of times and fluxes
    v += [2.0 ** k for k in range(-1074, 1024, 3)] + [-(2.0 ** k) for k in range(-80, 80)]
    v += [np.nextafter(2.0 ** k, np.inf) for k in range(-200, 200, 3)]
    v += [np.nextafter(2.0 ** k, 0.0) for k in range(-200, 200, 3)]
    v += [0.0, -0.0, 0.1, 0.2, 0.3, 1 / 3, 2 / 3, 1e23, 9007199254740993.0, 5e-324, 2.2250738585072014e-308,
          1.7976931348623157e308, 123.456, 1e-7, 0.001, -0.2, 1.2, 1.0, 100.0]
    return [float(x) for x in v]


def test_display_and_exponent_formats_match_rust(driver):
    vals = _values()
    out = subprocess.run([str(driver)] + [repr(x) for x in vals], capture_output=True, text=True,
                         check=True).stdout.splitlines()
    assert len(out) == len(vals)
    bad = [(x, line) for x, line in zip(vals, out)
           if line != f"{rust_disp(x)}|{rust_e(x, 15)}|{rust_e(x, 10)}"]
    assert not bad, bad[:5]
