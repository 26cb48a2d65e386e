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


def test_source_shards_cover_and_are_compact():
    case = wakes.rotor_sheet(40, seed=4, targets=100)
    m = len(case["starts"])
    for world in (1, 2, 5):
        parts = shard.source_shards(case["starts"], case["directions"], case["lengths"], world)
        assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(m))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
        assert all(np.all(np.diff(p) > 0) for p in parts)
    with pytest.raises(ValueError):
        shard.source_shards(case["starts"], case["directions"], case["lengths"], 0)


def _oracle_evaluator(model):
    """The CPU oracle's exact direct sum as a shard evaluator (torch tensors, as the GPU evaluator returns)."""
    from oracle import oracle as O

    def evaluate(points, starts, directions, lengths, gamma, radius):
        u, flags = O.direct_sum(points, starts, directions, lengths, gamma, radius, model,
                                (np.zeros(len(points) + 1, dtype=np.int64), np.zeros(0, dtype=np.int64)), "raise",
                                threads=1, return_flags=True)
        return torch.as_tensor(u), torch.as_tensor(flags)
    return evaluate


def _sharded_case():
    case = wakes.rotor_sheet(14, seed=7, targets=600)
    points = case["points"].copy()
    # one target on a segment: a singular pair that only the rank owning that segment sees
    points[5] = case["starts"][17] + 0.5 * case["lengths"][17] * case["directions"][17]
    return case, points


def _sharded_worker(rank, world, port, mode, result_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        case, points = _sharded_case()
        segments = tuple(case[k] for k in ("starts", "directions", "lengths", "gamma", "radius"))
        u, flags = shard.sharded_sum(_oracle_evaluator(case["model"]), points, segments, rank, world, mode)
        np.savez(result_path.replace(".npz", f"_{rank}.npz"), u=u.numpy(), flags=flags.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["sources", "targets"])
def test_sharded_sum_equals_the_single_rank_sum(tmp_path, mode):
    """The combined result of two gloo ranks, each evaluating its share with the oracle, equals the oracle's sum over
    the whole wake (to rounding: the ranks' partial sums add in another order), on both ranks, flags included."""
    from oracle import oracle as O
    world = 2
    path = str(tmp_path / "sharded.npz")
    mp.spawn(_sharded_worker, args=(world, _free_port(), mode, path), nprocs=world, join=True)
    case, points = _sharded_case()
    ref, ref_flags = O.direct_sum(points, *wakes.backend_args(case)[1:], (np.zeros(len(points) + 1, dtype=np.int64),
                                  np.zeros(0, dtype=np.int64)), "raise", return_flags=True)
    assert ref_flags[5] != 0 and ref_flags.sum() == ref_flags[5]
    for rank in range(world):
        got = np.load(str(tmp_path / f"sharded_{rank}.npz"))
        assert np.array_equal(got["flags"], ref_flags)
        ok = ref_flags == 0
        scale = np.abs(ref[ok]).max()
        np.testing.assert_allclose(got["u"][ok], ref[ok], rtol=0, atol=1e-13 * scale)
