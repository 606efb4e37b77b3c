"""Oracle answers for the benchmark's 1024-model batch (seed 1234).

bench.py evaluates the uneven 1024-model batch (lcurve-rs_b200/workloads.py
batch_models, seed 1234) on the GPU every run.  This script computes, once,
what the FP64 oracle (the restatement of the reference's CPU path) gives for
the same batch, so every bench run can check its own results:

  chisq     per model, unscaled (chisq_batch with scale = false), against
            data = the single_small curve at the model's times + 1% noise
            (workloads.batch_noise; here the curve is the oracle's, in the
            bench the engine's: they agree to ~1e-7, far inside the check)
  counters  line-of-sight searches (eclipse.rs:123-197 calls) and Roche
            potential / gradient evaluations of the eclipse search
            (potential.rs:110-127) over the whole batch

Usage: python tests/golden/make_bench_golden.py [THREADS]
Writes tests/golden/batch_1024_seed1234.json (about 20 minutes on 8 cores).
"""
import importlib
import json
import os
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

MODELS, SEED = 1024, 1234
OUT = HERE / f"batch_{MODELS}_seed{SEED}.json"


def main() -> None:
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    from oracle import oracle as O
    W = importlib.import_module("lcurve-rs_b200.workloads")
    specs = W.batch_models(n=MODELS, seed=SEED)
    offs = np.zeros(MODELS + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(t) for _, t in specs])
    times = np.concatenate([t for _, t in specs])
    t0 = time.time()
    fid = O.Model(text=W.single_small()[0]).light_curve(O.make_data(times, expose=0.001, ndiv=1),
                                                       nthreads=threads)["calc"]
    flux, sig = W.batch_noise(fid, SEED)
    data = O.make_data(times, expose=0.001, ndiv=1, flux=flux, ferr=sig, weight=1.0)
    print(f"fiducial curve at {len(times)} times: {time.time() - t0:.1f} s", flush=True)
    t0 = time.time()
    O.counters_reset()
    chisq = O.chisq_ragged([O.Model(text=s) for s, _ in specs], data, offs, scale=False, nthreads=threads)
    counters = O.counters()
    print(f"oracle chisq of {MODELS} models: {time.time() - t0:.1f} s; {counters}", flush=True)
    OUT.write_text(json.dumps({
        "workload": f"batch_models(n={MODELS}, seed={SEED}), data = single_small curve + 1% noise (batch_noise)",
        "workload_sha1": W.workload_key(specs),
        "chisq": [float(x) for x in chisq],
        "counters": counters,
    }, indent=0))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
