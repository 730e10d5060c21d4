"""Multi-rank host logic on CPU: two gloo ranks (spawned processes, 127.0.0.1).

Covers what the N-GPU benchmark relies on besides the kernels: the cost
balanced contiguous world shards (strong scaling), that a rank's shard is
exactly the full scene's worlds, and the max-over-ranks reductions used for
the timing and the run metrics.
"""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from newton_custom_contact_b200 import scenes
from newton_custom_contact_b200.distributed import max_over_ranks, partition_worlds, shard_range, world_costs


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    try:
        full, _ = scenes.scene_c2(seed=4, worlds=24, nmin=8, nmax=40, device="cpu")
        nb = np.diff(full._part["world_body_start"])
        a, b = shard_range(rank, world_size, nb)
        shard, _ = scenes.scene_c2(seed=4, worlds=24, nmin=8, nmax=40, device="cpu", world_range=(a, b))
        sel = (full.host("body_world") >= a) & (full.host("body_world") < b)
        same = np.array_equal(full.host("body_q")[sel], shard.host("body_q"))
        # every rank contributes its range, its own "elapsed ms" and metrics
        ranges = [None] * world_size
        dist.all_gather_object(ranges, (a, b))
        ms = max_over_ranks(10.0 + rank)
        metrics = max_over_ranks([0.001 * (rank + 1), 0.5 - rank])
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.array([same, ranges, ms, metrics, shard.body_count, int(sel.sum())], dtype=object),
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    res = [np.load(tmp_path / f"r{r}.npy", allow_pickle=True) for r in range(2)]
    for r in res:
        same, ranges, ms, metrics, nbody, nsel = r
        assert same and nbody == nsel
        assert ranges == [(ranges[0][0], ranges[0][1]), (ranges[1][0], ranges[1][1])]
        assert ranges[0][0] == 0 and ranges[0][1] == ranges[1][0] and ranges[1][1] == 24
        assert ms == 11.0
        assert metrics == [0.002, 0.5]


def test_partition_balances_cost():
    rng = np.random.default_rng(0)
    nb = rng.integers(8, 129, size=4096)
    for ws in (2, 4, 8):
        parts = partition_worlds(world_costs(nb), ws)
        assert parts[0][0] == 0 and parts[-1][1] == nb.size
        assert all(parts[i][1] == parts[i + 1][0] for i in range(ws - 1))
        loads = [world_costs(nb[a:b]).sum() for a, b in parts]
        assert max(loads) / min(loads) < 1.02


def test_partition_edge_cases():
    assert partition_worlds([1.0, 1.0], 2) == [(0, 1), (1, 2)]
    assert partition_worlds([100.0, 1.0, 1.0], 3) == [(0, 1), (1, 2), (2, 3)]
    with pytest.raises(ValueError):
        partition_worlds([1.0], 2)
    assert max_over_ranks(3.5) == 3.5  # no process group: identity


def _ws_worker(rank, world_size, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    from newton_custom_contact_b200.warmstart import allreduce_mean, moments

    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.Generator().manual_seed(0)
        x = torch.randn(1000, 5, generator=g) * torch.tensor([1.0, 2.0, 0.5, 3.0, 1.5]) + 0.3
        shard = x[rank::world_size]
        mean, std = moments(shard, dist.group.WORLD)
        grads = {"w": torch.full((3, 2), float(rank + 1)), "b": torch.tensor([10.0 * rank, 1.0])}
        allreduce_mean(grads, dist.group.WORLD)
        np.save(os.path.join(out_dir, f"ws{rank}.npy"),
                np.array([mean.numpy(), std.numpy(), grads["w"].numpy(), grads["b"].numpy(),
                          x.mean(0).numpy(), x.std(0).numpy()], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_warm_start_training_reductions_over_two_ranks(tmp_path):
    """Data-parallel warm-start training: normalisation moments over all ranks' samples and the
    gradient average, on two gloo ranks."""
    port = _free_port()
    mp.start_processes(_ws_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        mean, std, w, b, full_mean, full_std = np.load(tmp_path / f"ws{r}.npy", allow_pickle=True)
        np.testing.assert_allclose(mean, full_mean, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(std, full_std, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(w, np.full((3, 2), 1.5))
        np.testing.assert_allclose(b, np.array([5.0, 1.0]))
