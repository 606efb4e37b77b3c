"""The multi-rank logic of bench.py on CPU: two gloo ranks.

Each rank evaluates its own batch (weak scaling, seed 1234 + rank); the only
collective is the timing reduction, the slowest rank's step time; rank 0
alone runs the reference arm.
"""
import importlib
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        ms = [700.0, 950.0][rank]
        out[rank] = bench.max_over_ranks(ms, "cpu")
    finally:
        dist.destroy_process_group()


def test_timing_is_the_slowest_rank_and_value_is_weak_scaled():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1] == 950.0
    import bench
    assert bench.weak_value(world, 1024, 950.0) == pytest.approx(2 * 1024 / 0.95)
    assert bench.max_over_ranks(3.0, "cpu") == 3.0  # no process group: the rank's own value


def test_ranks_get_independent_batches():
    W = importlib.import_module("lcurve-rs_b200.workloads")
    a = W.batch_models(n=4, seed=1234 + 0)
    b = W.batch_models(n=4, seed=1234 + 1)
    assert [t for t, _ in a] != [t for t, _ in b]


def test_reference_arm_runs_on_rank_0_only(capsys):
    import bench

    class Args:
        pass
    assert bench.run_reference(Args(), rank=1, world=2) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the oracle on the host cores) prints one JSON
    line with the metric, unit and config of the GPU arm, its own cpu_baseline
    and an e2e with no device transfers."""
    import json
    import subprocess
    import sys

    from conftest import ROOT
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-sample", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    import bench
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["config"]["workload"].startswith("batch_1024")
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["kind"] == "port" and cpu["cores"] >= 1 and cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_mcmc_defaults_are_the_full_configuration(monkeypatch):
    """With no flags the MCMC comparison runs the full configuration (1M
    training curves, 300 epochs, 20000 steps); --mcmc-quick the reduced one;
    --tuning takes three launch-shape integers."""
    import bench
    monkeypatch.setattr("sys.argv", ["bench.py"])
    a = bench.parse()
    assert (a.mcmc_curves, a.mcmc_epochs, a.mcmc_steps) == (1048576, 300, 20000)
    monkeypatch.setattr("sys.argv", ["bench.py", "--mcmc-quick", "--tuning", "0,1,0"])
    a = bench.parse()
    assert (a.mcmc_curves, a.mcmc_epochs, a.mcmc_steps) == (524288, 250, 3000)
    assert [int(v) for v in a.tuning.split(",")] == [0, 1, 0]
