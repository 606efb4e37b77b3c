"""The index-checking build (LCURVE_DEBUG_BOUNDS, `make bounds`): every
device-side array index of the element, eclipse, flux and epilogue kernels is
checked against its array's size, an out-of-range access is skipped and
reported as LCB_ERR_DEVICE_CHECK instead of reading or writing out of range.
Here it runs the light-curve path's main shapes in a separate process
(LCB_LIBRARY selects the library) and must report no violation and give the
normal build's results."""
import json
import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

BOUNDS = ROOT / "lcurve-rs_b200" / "liblcurve_b200_bounds.so"

SCRIPT = r"""
import importlib, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
lcb = importlib.import_module("lcurve-rs_b200")
W = importlib.import_module("lcurve-rs_b200.workloads")
out = {"lib": str(lcb._capi.LIB_PATH)}
g = lcb.Model(sys.argv[2]).light_curve(time1=-0.2, time2=1.2, ntime=500, expose=0.001, ndiv=1)
out["golden"] = g.flux.tolist()
text, t, e, nd = W.single_large(nlat1=30, nlat2=60, ntime=400, nrad=30, nspot=30)
out["large"] = lcb.Model(text=text).light_curve(times=t, expose=e, ndiv=nd).flux.tolist()
specs = W.batch_models(n=8, seed=3, nlat1=(20, 40), nlat2=(30, 60), ntime=(100, 200))
models = [lcb.Model(text=s) for s, _ in specs]
offs = np.cumsum([0] + [len(t) for _, t in specs])
data = lcb.make_data(np.concatenate([t for _, t in specs]), flux=0.02, ferr=0.001, weight=1.0)
out["ragged"] = lcb.chisq_batch_ragged(models, data, offs, scale=True)[0].tolist()
B = lcb.Batch(models, data, offs)
B.run(scale=False)
out["resident"] = B.results()[0].tolist()
print(json.dumps(out))
"""


def _run(lib=None):
    env = dict(os.environ)
    env.pop("LCB_LIBRARY", None)
    if lib:
        env["LCB_LIBRARY"] = str(lib)
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT), str(GOLDEN / "test_model.dat")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_index_checking_build_finds_nothing_and_agrees():
    if not BOUNDS.exists():
        pytest.skip("liblcurve_b200_bounds.so not built (make -C lcurve-rs_b200 bounds)")
    checked = _run(BOUNDS)
    assert pathlib.Path(checked["lib"]).name == BOUNDS.name
    normal = _run()
    for key in ("golden", "large", "ragged", "resident"):
        a, b = np.array(checked[key]), np.array(normal[key])
        assert np.all(np.isfinite(a)), key
        assert np.allclose(a, b, rtol=1e-12, atol=0), key
