#!/usr/bin/env python
"""Benchmark: model evals/s of the 1024-model uneven chi-squared batch.

One step = one evaluation of a batch of 1024 models (per GPU) with uneven grid
sizes (nlat1f U{30..300}, nlat2f U{30..500}) and time counts (ntime
U{200..5000}): grids, FP64 Roche eclipses, continuum, FP32 flux sum over all
elements x times, chi-squared.  Inputs are seeded synthetic models and noisy
data (lcurve-rs_b200/workloads.py).

  value : device-resident throughput -- data uploaded once, each step replays
          the captured launch sequence (lcb_batch_run); CUDA events on the
          library's stream, max over ranks.
  e2e   : the same batch through lcb_chisq_batch_ragged with the inputs in
          pinned host memory: host planning, H2D of tables and data, kernels,
          D2H of the results, every step.

  mcmc  : (1 GPU) the surrogate pipeline -- light curves generated by the
          engine, the BF16 tensor-core MLP trained on them, then 256-walker
          delayed-acceptance MCMC against plain engine MCMC from one burned-in
          ensemble: ESS/s of each, surrogate error, posterior agreement.
          Default: the full configuration (1M curves, 300 epochs, 20000
          steps; about 12 minutes); --mcmc-quick runs a reduced one (524k
          curves, 3000 steps).  Headline: ESS/s of delayed acceptance over
          plain MCMC with the same (KDE) move.

  --autotune : tune the resident batch's launch shapes before timing (the
          default run uses the planner's heuristics).

  --train-profile K : only the surrogate's training step (8192 curves), K
          steps after --warmup, one JSON line (the profiling entry point).

Multi-GPU (torchrun): weak scaling, each rank evaluates its own 1024-model
batch (seed 1234 + rank); no collective on the data path, only the timing
reduction.  `--impl reference` times the CPU oracle (the FP64 restatement of
the reference's Rayon path) on the host cores instead.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib
import json
import os
import pathlib
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "model evals/s (1024-model batch) & MCMC ESS/s, surrogate-DA vs plain"
UNIT = "model evals/s"
FLUX_FLOPS_PER_EVAL = 17     # dot 5 + limb darkening 9 + product 2 + accumulate 1
POT_FLOPS_PER_EVAL = 22      # one Roche potential (or gradient) evaluation


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--models", type=int, default=1024)
    p.add_argument("--cpu-sample", type=int, default=0, help="models per CPU-baseline step (0 = host threads)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    # surrogate delayed-acceptance MCMC (256 walkers; 1 GPU)
    p.add_argument("--no-mcmc", action="store_true")
    p.add_argument("--mcmc-quick", action="store_true",
                   help="reduced run: 524k training curves, 250 epochs, 3000 steps (default: the full size, "
                        "1M curves, 300 epochs, 20000 steps)")
    p.add_argument("--mcmc-curves", type=int, default=1048576)
    p.add_argument("--mcmc-epochs", type=int, default=300)
    p.add_argument("--mcmc-steps", type=int, default=20000)
    p.add_argument("--mcmc-burn", type=int, default=500)
    p.add_argument("--mcmc-substeps", type=int, default=2)
    p.add_argument("--mcmc-bandwidth", type=float, default=0.6, help="KDE bandwidth in units of Scott's factor")
    p.add_argument("--mcmc-refine", type=int, default=262144,
                   help="curves for sharpening the surrogate near the burned-in ensemble (0: none)")
    p.add_argument("--autotune", action="store_true",
                   help="tune the resident batch's launch shapes (lcurve-rs_b200/autotune.py) before timing")
    p.add_argument("--tuning", default="", metavar="CHUNKS,SPLIT,BPS",
                   help="fixed launch shapes of the resident batch (lcb_batch_set_tuning; 0 = heuristic), "
                        "e.g. 0,1,0 for one scan thread per element in a small profiling case")
    p.add_argument("--train-profile", type=int, default=0, metavar="K",
                   help="time K surrogate training steps (8192 curves) alone, print one JSON line and exit")
    a = p.parse_args()
    if a.mcmc_quick:
        a.mcmc_curves, a.mcmc_epochs, a.mcmc_steps = 524288, 250, 3000
    return a


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i",
                 str(self.device), "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload(lcb, W, n, seed):
    specs = W.batch_models(n=n, seed=seed)
    models = [lcb.Model(text=s) for s, _ in specs]
    offs = np.zeros(n + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(t) for _, t in specs])
    times = np.concatenate([t for _, t in specs])
    # data = the single_small model's curve at each model's times + 1% noise
    fid_text = W.single_small()[0]
    fid = [lcb.Model(text=fid_text) for _ in range(n)]
    tmpl = lcb.make_data(times, expose=0.001, ndiv=1, flux=1.0, ferr=1.0, weight=1.0)
    _, fflux, _ = lcb.chisq_batch_ragged(fid, tmpl, offs, scale=False, want_calc=True)
    flux, sig = W.batch_noise(fflux, seed)
    data = lcb.make_data(times, expose=0.001, ndiv=1, flux=flux, ferr=sig, weight=1.0)
    return specs, models, data, offs


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_sample(specs, data, offs, sel, nthreads):
    """The oracle's chi-squared of the models `sel` on all host threads, with
    the reference's Rayon loops (models, and within each model its times, in
    parallel; threads that run out of models help with other models' times).
    Returns (chisq, wall-clock models/s, steady-state models/s).  Steady state
    is the rate of a batch long enough to keep every thread busy, as the
    reference's chisq_batch over 1024 models is: models x threads / process
    CPU seconds.  A short sample's own wall clock undercounts it, since its
    last models run while other threads idle."""
    import resource

    from oracle import oracle as O
    oms = [O.Model(text=specs[i][0]) for i in sel]
    parts, o2 = [], [0]
    for i in sel:
        parts.append(data[offs[i]:offs[i + 1]])
        o2.append(o2[-1] + offs[i + 1] - offs[i])
    d = np.concatenate(parts)
    r0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    chi = O.chisq_ragged(oms, d, o2, scale=False, nthreads=nthreads)
    wall = time.perf_counter() - t0
    r1 = resource.getrusage(resource.RUSAGE_SELF)
    cpu = (r1.ru_utime - r0.ru_utime) + (r1.ru_stime - r0.ru_stime)
    return chi, len(sel) / wall, len(sel) * nthreads / max(cpu, 1e-9)


def cpu_description(nthreads) -> dict:
    from oracle import oracle as O
    return {"cores": nthreads, "cpu_model": O.host_cpu(),
            "build": "oracle/lcurve_oracle.cpp, g++ -O3 -march=native -ffp-contract=off, built on this host"}


def bench_golden(models: int, seed: int):
    """Committed oracle answers for this batch (tests/golden/make_bench_golden.py), if any."""
    p = ROOT / "tests" / "golden" / f"batch_{models}_seed{seed}.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text())
    except (ValueError, OSError):
        return None


def traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(kernel, {}).get("dram_bytes_per_launch_full_workload")
    except (ValueError, OSError):
        return None


def spot_stream_timing(lcb, specs, data, offs, steps=3):
    """Wall-clock ms of lcb_chisq_batch_ragged on these models with a bright
    spot (add_spot = 1): every call with the same q (the planner's memo of the
    gas-stream end point hits) and every call with new q values (every
    model's Bulirsch-Stoer stream integration runs on the host,
    crates/roche/src/stream.rs:82-145)."""
    models = []
    for text, _ in specs:
        m = lcb.Model(text=text)
        m.set_comp("add_spot", "1")
        models.append(m)
    q0 = np.array([m.q for m in models])
    out = {}
    for case in ("same_q", "new_q"):
        ms = []
        for s in range(steps + 1):
            if case == "new_q":
                for m, q in zip(models, q0):
                    m.q = q * (1.0 + 1e-9 * (s + 1))
            t0 = time.perf_counter()
            chi, _, _ = lcb.chisq_batch_ragged(models, data, offs, scale=False)
            if s:
                ms.append((time.perf_counter() - t0) * 1e3)
        out[case + "_ms"] = float(np.median(ms))
    out["stream_ms_per_call"] = out["new_q_ms"] - out["same_q_ms"]
    out["models"] = len(models)
    out["failed_models"] = int(np.count_nonzero(~np.isfinite(chi)))
    return out


def run_reference(args, rank, world):
    """The reference arm: the CPU path (the oracle, the FP64 restatement of the
    reference's Rayon chisq_batch, built for this host's CPU) on the same
    1024-model batch and data.  Each timed step evaluates 2 x threads models,
    rotating through the batch; warm-up steps a few."""
    if rank != 0:
        return
    W = importlib.import_module("lcurve-rs_b200.workloads")
    from oracle import oracle as O
    O.use_native()
    nthreads = host_threads()
    sample = args.cpu_sample or 2 * nthreads
    warm = max(1, nthreads // 4)
    specs = W.batch_models(n=args.models, seed=1234)
    n = len(specs)
    offs = np.zeros(n + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(t) for _, t in specs])
    times = np.concatenate([t for _, t in specs])
    # the b200 arm's data: the single_small curve at every model's times + 1% noise; the
    # curve is evaluated (by the CPU path) only where a sampled model needs it
    sels = [[(s * warm + k) % n for k in range(warm)] for s in range(args.warmup)]
    sels += [[(s * sample + k) % n for k in range(sample)] for s in range(args.steps)]
    need = np.zeros(times.shape[0], dtype=bool)
    for i in {i for sel in sels for i in sel}:
        need[offs[i]:offs[i + 1]] = True
    fid = np.zeros(times.shape[0])
    fid[need] = O.Model(text=W.single_small()[0]).light_curve(O.make_data(times[need]), nthreads=nthreads)["calc"]
    flux, sig = W.batch_noise(fid, 1234)
    data = O.make_data(times, expose=0.001, ndiv=1, flux=flux, ferr=sig, weight=1.0)
    steady, wall = [], []
    for s, sel in enumerate(sels):
        _, rw, rs = cpu_sample(specs, data, offs, sel, nthreads)
        if s >= args.warmup:
            wall.append(rw)
            steady.append(rs)
    v = float(np.mean(steady))
    cpu = cpu_description(nthreads)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sample / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"batch_{args.models}: uneven models (nlat1f U{{30..300}}, nlat2f U{{30..500}}, "
                               f"ntime U{{200..5000}}, q/iangle/r1/t1/t2 uniform), seed 1234",
                   "sample_models_per_step": sample, "warmup_models_per_step": warm,
                   "wall_clock_models_per_s": float(np.mean(wall))},
        "cpu_baseline": {"value": v, "unit": UNIT, "kind": "port", **cpu,
                         "sample": f"{sample} models per step rotating through the 1024-model batch "
                                   f"({args.steps * sample} models), all host threads, nested model/time "
                                   "parallelism as the reference's Rayon chisq_batch; value = steady-state rate "
                                   "(models x threads / process CPU s), wall-clock rate in config"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "mcmc": {"skipped": "the MCMC comparison runs the GPU engine and surrogate; the reference arm times "
                            "the CPU light-curve path only"},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, device) -> float:
    """The largest value of x over the ranks of the default process group
    (each rank's own value when there is none): step times are reported as
    the slowest rank's."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(world: int, models_per_rank: int, ms_max: float) -> float:
    """Whole-job model evals/s: every rank evaluates its own batch, in the slowest rank's time."""
    return world * models_per_rank / (ms_max / 1e3)


def run_train_profile(args, lcb):
    """K training steps of the surrogate network (5 -> 4 x 512 -> 256, 8192
    curves a step: forward, backward, Adam) on seeded synthetic inputs, after
    --warmup steps; host wall clock around the stream (one sync each side).
    The launch-list profile of the surrogate's kernels runs this."""
    import torch

    S = importlib.import_module("lcurve-rs_b200.surrogate")
    sur = S.Surrogate()
    b = sur.max_batch
    g = torch.Generator(device=sur.dev).manual_seed(0)
    x = torch.rand(b, len(S.PARAMS), device=sur.dev, generator=g) * 2 - 1
    y = torch.randn(b, sur.n_phase, device=sur.dev, generator=g)
    torch.cuda.synchronize()

    def step():
        lcb._capi.check_mlp(sur.L.lcb_mlp_train_step(sur._h, ctypes.c_void_p(x.data_ptr()),
                                                     ctypes.c_void_p(y.data_ptr()), b, 1e-3, 0.9, 0.999, 1e-8, 0.0))

    for _ in range(args.warmup):
        step()
    lcb._capi.check_mlp(sur.L.lcb_mlp_sync(sur._h))
    t0 = time.perf_counter()
    for _ in range(args.train_profile):
        step()
    lcb._capi.check_mlp(sur.L.lcb_mlp_sync(sur._h))
    dt = (time.perf_counter() - t0) / max(args.train_profile, 1)
    n_par = len(S.PARAMS)
    flops = 6 * b * ((n_par + 7) // 8 * 8 * sur.width + (sur.n_hidden - 1) * sur.width ** 2 + sur.width * sur.n_phase)
    print(json.dumps({"surrogate_train_step_ms": dt * 1e3, "batch": b, "steps": args.train_profile,
                      "warmup": args.warmup, "gemm_tflops_6bp": flops / dt / 1e12,
                      "network": f"{n_par} -> {sur.n_hidden} x {sur.width} (GELU) -> {sur.n_phase}"}))


def likelihood_roughness(eng) -> dict:
    """The engine's chi-squared along short lines through the truth (61 points
    over +-0.01 in q, +-0.2 deg in iangle): the residual std about a quartic
    fit is the non-smooth part of the likelihood (the discrete grid's elements
    entering and leaving eclipse), which no smooth surrogate can learn."""
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    out = {}
    for k, name, h in ((0, "q", 0.01), (1, "iangle", 0.2)):
        x = np.linspace(-1.0, 1.0, 61)
        th = np.repeat(S.TRUTH[None, :], len(x), axis=0)
        th[:, k] += h * x
        chi = eng.chisq(th)
        res = chi - np.polyval(np.polyfit(x, chi, 4), x)
        out[name] = {"half_width": h, "residual_std": float(res.std()), "chisq_range": float(np.ptp(chi))}
    return out


def run_mcmc(args, lcb):
    """Surrogate delayed-acceptance MCMC against plain engine MCMC: 256
    walkers on the fixed 256-phase problem (fiducial curve + 1% noise), all
    samplers started from one burned-in ensemble; ESS/s over the sampling
    loops.  Plain samplers: the stretch move (the reference fitter's emcee
    default) and the KDE move; the delayed-acceptance sampler screens KDE
    moves with the surrogate."""
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    M = importlib.import_module("lcurve-rs_b200.mcmc")
    W = importlib.import_module("lcurve-rs_b200.workloads")
    setup = S.CurveSetup()
    n, hold = args.mcmc_curves, 4096
    t0 = time.perf_counter()
    theta = S.sample_prior(n + hold, seed=1)
    curves = S.generate_curves(setup, theta)
    gen_s = time.perf_counter() - t0
    sur = S.Surrogate()
    losses = sur.fit(theta[:n], curves[:n], epochs=args.mcmc_epochs)
    train_global_s = sur.train_seconds
    ok = np.isfinite(curves[n:]).all(axis=1)
    rel = S.scaled_rel_error(sur.predict(theta[n:][ok]), curves[n:][ok])

    fid = S.CurveEngine(setup).curves(S.TRUTH[None, :])[0]
    data = W.noisy_data(setup.times, fid, setup.expose, setup.ndiv, seed=42)
    eng = S.CurveEngine(setup, data=data)
    sur.bind_data(data)
    p0 = M.initial_walkers(256, S.TRUTH, seed=3)
    burn = M.run_delayed(eng, sur, p0, args.mcmc_burn, seed=4, substeps=32)
    start = burn.chain[-1]
    sample = start[:128]
    dchi_global = eng.chisq(sample) - sur.chisq(sample)
    refine_s = 0.0
    if args.mcmc_refine:  # more training where the sampler sits; the samplers stay exact
        refine_s = S.refine_near(sur, setup, start, theta[:n], curves[:n], n=args.mcmc_refine, widen=2.5,
                                 epochs=100, lr=1e-3)
    bw, k = args.mcmc_bandwidth, args.mcmc_substeps
    runs = {
        "plain_stretch": M.run_plain(eng, start, args.mcmc_steps, seed=5),
        "plain_kde": M.run_plain(eng, start, args.mcmc_steps, seed=5, move="kde", bandwidth=bw),
        "da_kde": M.run_delayed(eng, sur, start, args.mcmc_steps, seed=5, substeps=k, move="kde", bandwidth=bw),
    }
    ess = {name: M.ess(r, burn=0.0) for name, r in runs.items()}
    rate = {name: ess[name][0] / r.seconds for name, r in runs.items()}
    post = {name: M.posterior_summary(r, burn=0.0) for name, r in runs.items()}
    ref = post["plain_stretch"]
    shift = {name: max(abs(p[q][0] - ref[q][0]) / ref[q][1] for q in ref) for name, p in post.items()}
    dchi = eng.chisq(sample) - sur.chisq(sample)
    overhead = gen_s + train_global_s + refine_s  # curves, training and refinement
    da = runs["da_kde"]
    return {
        "headline": "speedup_vs_plain_same_move",
        "speedup_vs_plain_same_move": rate["da_kde"] / rate["plain_kde"],
        "target_speedup": 5.0,
        "ess_per_s": rate,
        "speedup_vs_plain_stretch": rate["da_kde"] / rate["plain_stretch"],
        # of the moves the surrogate accepted, the share the engine accepted too; with a surrogate
        # chi-squared error of std s (independent at the two points) it is E[min(1, exp(N(0, s^2/2)))]
        "da_stage2_acceptance": da.accepted / max(da.stage1_pass, 1),
        "likelihood_roughness": likelihood_roughness(eng),
        "ess_per_s_da_incl_training": ess["da_kde"][0] / (runs["da_kde"].seconds + overhead),
        "ess": {name: e[0] for name, e in ess.items()},
        "tau": {name: e[1].tolist() for name, e in ess.items()},
        "seconds": {**{name: r.seconds for name, r in runs.items()}, "curve_generation": gen_s,
                    "training": train_global_s, "refine": refine_s, "burn_in": burn.seconds},
        "engine_evals": {name: r.engine_evals for name, r in runs.items()},
        "acceptance": {name: r.acceptance for name, r in runs.items()},
        "posterior": post, "max_mean_shift_vs_plain_stretch_in_sigma": shift,
        "surrogate": {"network": "5 -> 4 x 512 (GELU) -> 256, BF16 tcgen05 kernels, FP32 accumulation",
                      "train_curves": n, "epochs": args.mcmc_epochs, "final_loss": losses[-1],
                      "holdout_scaled_rel_err": {"median": float(np.median(rel)),
                                                 "p99": float(np.quantile(rel, 0.99)), "max": float(rel.max())},
                      "posterior_chisq_minus_engine": {"mean": float(-dchi.mean()), "std": float(dchi.std())},
                      "posterior_chisq_minus_engine_before_refine": {"mean": float(-dchi_global.mean()),
                                                                     "std": float(dchi_global.std())},
                      "refine": {"curves": args.mcmc_refine, "seconds": refine_s,
                                 "how": "Gaussian of the burned-in ensemble, covariance x 2.5^2, 100 epochs mixed "
                                        "with as many global rows (surrogate.refine_near)"}},
        "config": {"walkers": 256, "steps": args.mcmc_steps, "burn_in_steps": args.mcmc_burn,
                   "da_substeps": k, "kde_bandwidth_x_scott": bw, "phases": setup.n_phase, "stretch_a": 2.0,
                   "likelihood": "-chisq/2, chisq_batch scale=True, uniform prior box of the 1024-model batch",
                   "data": "fiducial single_small curve at 256 phases + 1% Gaussian noise, seed 42",
                   "timing": "wall clock of each sampling loop (host-driven; engine and surrogate on the GPU)"},
    }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    lcb = importlib.import_module("lcurve-rs_b200")
    W = importlib.import_module("lcurve-rs_b200.workloads")
    lcb.set_device(f"cuda:{local}")
    if args.train_profile:
        run_train_profile(args, lcb)
        return
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    lcb.set_stream(stream.cuda_stream)  # the library's work and the timing events share this stream

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    specs, models, data, offs = build_workload(lcb, W, args.models, 1234 + rank)
    B = lcb.Batch(models, data, offs)
    tuned = None
    if args.tuning:
        B.set_tuning(*(int(v) for v in args.tuning.split(",")))
    if args.autotune:  # off by default: the heuristics' launch shapes
        tuned = importlib.import_module("lcurve-rs_b200.autotune").autotune(B, scale=False, repeats=1)
    st = B.stats()
    for _ in range(args.warmup):
        B.run(scale=False)

    # ---- device-resident value
    barrier()
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            B.run(scale=False)  # CUDA-graph replay
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1) / args.steps
        # per-kernel device times: the same launch sequence issued directly with CUDA events
        # between the kernels on this stream (events inside a graph carry no timing)
        stage_names = ["phase", "elements", "roche", "aux", "flux", "epilogue"]
        stage_acc = np.zeros(len(stage_names))
        for _ in range(args.steps):
            s = B.profile(scale=False)
            stage_acc += np.array([s[k] for k in stage_names])
        counts = B.search_counts()
        barrier()
    st = B.stats()
    chi, _, _ = B.results()
    ms_max = max_over_ranks(ms, "cuda")
    value = weak_value(world, args.models, ms_max)
    stage = stage_acc / args.steps

    # ---- end-to-end through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(data.nbytes, dtype=torch.uint8, pin_memory=True)
        pdata = pinned.numpy().view(lcb.DATUM_DTYPE)
        pdata[:] = data
        lcb.chisq_batch_ragged(models, pdata, offs, scale=False)  # warm the transient buffers
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            c2, _, _ = lcb.chisq_batch_ragged(models, pdata, offs, scale=False)
        e1.record(stream)
        barrier()
        wall = (time.perf_counter() - w0) / args.steps * 1e3
        h2d, d2h = lcb.transfer_bytes()
        e2e_ms = max_over_ranks(max(e0.elapsed_time(e1) / args.steps, wall), "cuda")
        # a tuned batch differs from the transient (heuristic) plan in FP32 summation order only
        same = bool(np.allclose(c2, chi, rtol=1e-4 if tuned else 1e-9, equal_nan=True))
        e2e = {"value": weak_value(world, args.models, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms, "matches_resident": same}

    # ---- bright-spot models: the host's gas-stream integration when q changes every call
    spot = None
    if not args.no_e2e and world == 1:
        spot = {"batch_1024": spot_stream_timing(lcb, specs, pdata, offs),
                "batch_16": spot_stream_timing(lcb, specs[:16], pdata[:offs[16]], offs[:17])}

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    # ---- parity of this run's batch against the oracle's committed answers (all models)
    golden = bench_golden(args.models, 1234 + rank)
    parity = {}
    if golden is not None:
        if W.workload_key(specs) == golden["workload_sha1"]:
            ref = np.asarray(golden["chisq"])
            parity["batch_vs_oracle"] = {
                "models": int(ref.size), "max_rel_err_chisq": float(np.max(np.abs(chi - ref) / np.abs(ref))),
                "searches": int(counts["searches"]), "oracle_searches": int(golden["counters"]["fblink"]),
                "source": "tests/golden/batch_1024_seed1234.json (oracle, tests/golden/make_bench_golden.py)"}

    # ---- roofline of the dominant kernel
    p64 = lcb.fma_peak_tflops(True)
    p32 = lcb.fma_peak_tflops(False)
    # FP64 work of the Roche search, two ways: as executed on the device (potential and
    # gradient evaluations plus miss-proof nodes, each a potential and a gradient evaluation),
    # and as the reference's algorithm counts it (the oracle's potential and gradient
    # evaluations for this batch; the device proves most misses without them)
    roche_flops = (counts["pot_evals"] + counts["dpot_evals"] + 2 * counts["bound_nodes"]) * POT_FLOPS_PER_EVAL
    roche_alg = None
    if golden is not None and parity:
        roche_alg = (golden["counters"]["rpot"] + golden["counters"]["drpot"]) * POT_FLOPS_PER_EVAL
    flux_flops = st["element_evals"] * FLUX_FLOPS_PER_EVAL
    kernels = {
        "k_roche": {"ms": stage[2], "flops": roche_alg or roche_flops, "peak": p64, "pipe": "fp64",
                    "work": "reference-algorithm potential evaluations (oracle count) x 22" if roche_alg
                    else "executed potential and gradient evaluations (2 per miss-proof node) x 22"},
        "k_flux": {"ms": stage[4], "flops": flux_flops, "peak": p32, "pipe": "fp32",
                   "work": "element-evals x 17"},
    }
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    k = kernels[dom]
    ach = k["flops"] / (k["ms"] / 1e3) / 1e12
    tf = lambda fl, ms: fl / (ms / 1e3) / 1e12 if ms else None  # noqa: E731
    roof = {"kernel": dom, "bound": k["pipe"], "achieved": ach, "peak": k["peak"], "unit": "TFLOP/s",
            "frac": ach / k["peak"] if k["peak"] else None, "traffic": traffic_from_profiles(dom),
            "work": k["work"],
            "peak_source": f"measured {k['pipe'].upper()} FMA peak of this GPU (k_fma_peak); "
                           "MEASURED_PEAKS.json has no FP32/FP64 figure",
            "k_roche_executed": {"achieved_tflops": tf(roche_flops, stage[2]),
                                 "frac": tf(roche_flops, stage[2]) / p64 if stage[2] and p64 else None},
            "other": {n: {"ms": v["ms"], "achieved_tflops": tf(v["flops"], v["ms"]), "peak_tflops": v["peak"],
                          "work": v["work"]} for n, v in kernels.items()}}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.use_native()
        nthreads = host_threads()
        sample = args.cpu_sample or 2 * nthreads
        sel = list(range(min(sample, len(specs))))
        ochi, rate_wall, rate = cpu_sample(specs, data, offs, sel, nthreads)
        cpu = {"value": rate, "unit": UNIT, "kind": "port", **cpu_description(nthreads),
               "sample": f"first {len(sel)} models of the batch, all host threads, nested model/time parallelism "
                         "as the reference's Rayon chisq_batch; value = steady-state rate (models x threads / "
                         "process CPU s)", "wall_clock_models_per_s": rate_wall}
        parity["sample_vs_oracle"] = {"models": len(sel),
                                      "max_rel_err_chisq": float(np.max(np.abs(chi[sel] - ochi) / np.abs(ochi)))}

    mcmc = None
    if world == 1 and not args.no_mcmc:
        mcmc = run_mcmc(args, lcb)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 eclipses + f32 flux", "data": "synthetic",
        "config": {"workload": f"batch_{args.models}: uneven models (nlat1f U{{30..300}}, nlat2f U{{30..500}}, "
                               f"ntime U{{200..5000}}, q/iangle/r1/t1/t2 uniform), seed 1234+rank",
                   "models_per_gpu": args.models, "elements_per_step": st["elements"],
                   "subphases_per_step": st["subphases"], "element_evals_per_step": st["element_evals"],
                   "roche_eclipsed_elements": st["roche_elements"], "roche_search": counts,
                   "flux_units": st["flux_units"],
                   **({"autotuned": tuned} if tuned else {}),
                   "stage_ms": dict(zip(stage_names, [float(x) for x in stage])),
                   "l2": "inputs larger than L2 (element arrays > 10 GB per step)",
                   "parallelism": f"weak, {world} independent batches"},
        "roofline": roof,
        "parity": parity or None,
        "spot_stream": spot,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": 6 * args.steps,
        "clocks": clk.summary(),
        "mcmc": mcmc if mcmc is not None else {"skipped": "multi-GPU run or --no-mcmc; the MCMC comparison runs on 1 GPU"},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
