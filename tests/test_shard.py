"""Sharding over the GPUs of a node (openfawe_b200.shard): partitions on the CPU and the gather path as world-size-2
``gloo`` process groups (the same calls NCCL runs between GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from openfawe_b200 import shard, wakes


def test_morton_order_and_target_shards():
    case = wakes.rotor_sheet(60, seed=3, targets=5000)
    points = case["points"]
    order = shard.morton_order(points)
    assert np.array_equal(np.sort(order), np.arange(len(points)))
    for world in (1, 2, 3, 8):
        parts = shard.target_shards(points, world)
        assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(len(points)))
        sizes = [len(p) for p in parts]
        assert max(sizes) - min(sizes) <= 1
        if world > 1:
            # Morton ranges are spatially compact: their boxes add up to far less than the `world` near-whole boxes of
            # an unordered split
            whole = np.prod(np.ptp(points, axis=0))
            assert sum(np.prod(np.ptp(points[p], axis=0)) for p in parts) < 0.6 * world * whole
    assert [len(p) for p in shard.target_shards(np.zeros((0, 3)), 2)] == [0, 0]
    with pytest.raises(ValueError):
        shard.target_shards(points, 0)


def test_wake_shards_balance_and_cover():
    rng = np.random.default_rng(48)
    sizes = [(int(s), int(t)) for s, t in zip(np.exp(rng.uniform(np.log(5e3), np.log(4.1e5), 48)),
                                              np.exp(rng.uniform(np.log(2e3), np.log(20570), 48)))]
    for world in (1, 2, 4, 8):
        parts, load = shard.wake_shards(sizes, world)
        assert sorted(w for p in parts for w in p) == list(range(48))
        assert all(p == sorted(p) for p in parts)
        biggest = max(shard.wake_cost(*s) for s in sizes)
        # greedy largest-first: no rank exceeds the mean load by more than the largest wake
        assert load.max() <= load.mean() + biggest
        assert parts == shard.wake_shards(sizes, world)[0]  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, total, result_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        points = rng.normal(size=(total, 3))
        mine = shard.target_shards(points, world)[rank]
        # each rank's rows are a function of the target index, as its evaluation would be
        local = torch.as_tensor(np.column_stack((mine * 10.0, mine * 10.0 + 1, -mine.astype(np.float64))))
        full = shard.gather(local, mine, total)
        if rank == 0:
            np.save(result_path, full.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("total", [1001, 3])
def test_gather_reassembles_target_order(tmp_path, total):
    world = 2
    path = str(tmp_path / "full.npy")
    mp.spawn(_gather_worker, args=(world, _free_port(), total, path), nprocs=world, join=True)
    full = np.load(path)
    idx = np.arange(total, dtype=np.float64)
    np.testing.assert_array_equal(full, np.column_stack((idx * 10.0, idx * 10.0 + 1, -idx)))
