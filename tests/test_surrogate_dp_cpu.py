"""Data-parallel surrogate training's scheme on CPU: two gloo ranks.

Surrogate.fit(group=...) splits every global batch into equal contiguous
shards (surrogate.shard_rows) of a permutation all ranks share, averages the
ranks' mean-squared-error gradients with an all-reduce, and takes the same
Adam step everywhere.  Here a small FP64 torch network stands in for the
device network: after a few steps the data-parallel ranks must hold the
weights that one process training on the whole batches holds (1e-12), and
the same weights on both ranks.
"""
import importlib
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

STEPS, BATCH, N = 4, 64, 256


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    g = torch.Generator().manual_seed(0)
    x = torch.rand(N, 5, generator=g, dtype=torch.float64) * 2 - 1
    y = torch.sin(x @ torch.randn(5, 8, generator=g, dtype=torch.float64))
    return x, y


def _net():
    torch.manual_seed(1)
    return torch.nn.Sequential(torch.nn.Linear(5, 16), torch.nn.GELU(), torch.nn.Linear(16, 8)).double()


def _train(rank, world, group=None):
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    x, y = _problem()
    net = _net()
    opt = torch.optim.Adam(net.parameters(), lr=1e-2)
    perm = torch.randperm(N, generator=torch.Generator().manual_seed(2))
    for k in range(STEPS):
        idx = perm[S.shard_rows(k, BATCH, rank, world)]
        opt.zero_grad()
        torch.nn.functional.mse_loss(net(x[idx]), y[idx]).backward()  # mean over this shard
        if group is not None:
            import torch.distributed as dist
            for p in net.parameters():
                dist.all_reduce(p.grad, group=group)
                p.grad.div_(world)
        opt.step()
    return torch.cat([p.detach().ravel() for p in net.parameters()]).numpy()


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        out[rank] = _train(rank, world, dist.group.WORLD)
    finally:
        dist.destroy_process_group()


def test_shards_cover_each_global_batch_once():
    S = importlib.import_module("lcurve-rs_b200.surrogate")
    for world in (1, 2, 4):
        for k in range(3):
            rows = np.concatenate([np.arange(N)[S.shard_rows(k, BATCH, r, world)] for r in range(world)])
            assert np.array_equal(rows, np.arange(k * BATCH, (k + 1) * BATCH))


def test_data_parallel_ranks_take_the_whole_batch_step():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    single = _train(0, 1)
    assert np.array_equal(out[0], out[1])
    assert np.allclose(out[0], single, rtol=1e-12, atol=1e-14)
