"""Shared pytest configuration.

Markers:
  gpu — needs a CUDA device (run on a B200 with `pytest -m gpu`).
"""
import importlib
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def rust_e(x, prec):
    """Rust's {:.Ne} of an f64: N decimals, exponent without sign padding or zeros."""
    mant, exp = f"{x:.{prec}e}".split("e")
    return f"{mant}e{int(exp)}"


def rust_disp(x):
    """Rust's Display of an f64: the shortest round-trip digits (closest to x),
    positional, no trailing .0."""
    import numpy as np
    return np.format_float_positional(x, unique=True, trim="-")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def lcb():
    """The product package (directory lcurve-rs_b200/)."""
    return importlib.import_module("lcurve-rs_b200")


@pytest.fixture(scope="session")
def test_model_path():
    return GOLDEN / "test_model.dat"
