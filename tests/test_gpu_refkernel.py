"""The reference's own CUDA flux kernel (crates/lcurve-cuda/kernels/
flux_kernel.cu, compiled unmodified for sm_100a into oracle/_ref by
`make -C oracle ref`) on this GPU, fed the inputs its Rust host code prepares
(oracle/ref_gpu.py), as the GPU comparator of the flux stage.

* single_small: its light curve against the oracle's within the reference's
  own GPU-vs-CPU bound, 1e-3 (crates/lcurve-cuda/tests/gpu_correctness.rs:
  90-94), which its f32 phases and 3-pair eclipse lists need;
* single_large at full size (nlat 200/400, disc, rim, spot, 10,000 x 5): its
  kernel time against this engine's flux stage on the same model and times
  (CUDA events on one stream), printed for the record.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    from oracle import ref_gpu
    if not ref_gpu.available():
        pytest.skip("oracle/_ref/libref_flux.so not built (make -C oracle ref REF_ROOT=<reference checkout>)")
    return ref_gpu


def _ref_run(R, oracle, text, t, expose, ndiv):
    G = oracle.Model(text=text).built_grids(threads=16)
    run = R.Run(*R.prepare(text, t, expose, ndiv, G))
    return G, run


def test_reference_kernel_light_curve(R, oracle):
    W = importlib.import_module("lcurve-rs_b200.workloads")
    text, t, expose, ndiv = W.single_small()
    G, run = _ref_run(R, oracle, text, t, expose, ndiv)
    try:
        run.launch()
        got = run.result()
    finally:
        run.free()
    o = G.light_curve(oracle.make_data(t, expose=expose, ndiv=ndiv), nthreads=8)["calc"]
    err = float(np.max(np.abs(got - o) / np.abs(o)))
    print(f"reference CUDA kernel, single_small: max rel err vs oracle {err:.2e}")
    assert err < 1e-3


def test_reference_kernel_time_against_the_flux_stage(R, oracle, lcb):
    import torch
    W = importlib.import_module("lcurve-rs_b200.workloads")
    text, t, expose, ndiv = W.single_large()
    stream = torch.cuda.Stream()
    G, run = _ref_run(R, oracle, text, t, expose, ndiv)
    try:
        run.launch(stream.cuda_stream)  # warm-up
        ms = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run.launch(stream.cuda_stream)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        ref_flux = run.result()
    finally:
        run.free()
    d = lcb.make_data(t, expose=expose, ndiv=ndiv, ferr=1.0, weight=1.0)
    B = lcb.Batch([lcb.Model(text=text)], d, [0, d.shape[0]])
    B.run()
    prof = [B.profile() for _ in range(3)]
    flux_ms = min(p["flux"] for p in prof)
    total_ms = min(sum(p.values()) for p in prof)
    _, calc, _ = B.results(want_calc=True)
    print(f"single_large full size: reference flux_eval_kernel {min(ms):.2f} ms; this engine's flux stage "
          f"{flux_ms:.2f} ms ({min(ms) / flux_ms:.1f}x), whole evaluation incl. grids and eclipses {total_ms:.2f} ms")
    assert np.max(np.abs(ref_flux - calc) / np.abs(calc)) < 1e-3
