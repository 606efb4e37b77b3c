"""Regenerates the golden fixtures in this directory from the reference tree.

The reference (scope-ml/lcurve-rs) ships one true external golden for the
light-curve path: test_data/test_lc.dat, 500 fluxes that the original C++
lroche wrote for test_data/test_model.dat (times -0.2..1.2, expose 0.001,
ndiv 1; see the reference's tests/regression.rs:9-88).  Both files are copied
verbatim so the tests can run where the reference tree is absent.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
(REFERENCE_ROOT: the root of a checkout of the reference project.)
"""
import pathlib
import shutil
import sys

HERE = pathlib.Path(__file__).resolve().parent


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
    ref = pathlib.Path(sys.argv[1])
    for name in ("test_model.dat", "test_lc.dat"):
        shutil.copyfile(ref / "test_data" / name, HERE / name)
        print("wrote", HERE / name)


if __name__ == "__main__":
    main()
