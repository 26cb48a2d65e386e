"""Sharding of the induced-velocity sums over the GPUs of one node (one process per GPU).

Every target is independent, so the path shards without a collective on its data path:

* one wake: the segments (and so the tree and its moments) are replicated on every rank, the targets are split into
  contiguous ranges of their Morton order (spatially compact shards keep each rank's traversal coherent) of equal
  size; each rank evaluates its own range;
* a batch of wakes: wakes are assigned whole to ranks, largest first to the least-loaded rank (cost = segments x
  targets^(1/2) + targets, a stand-in for the tree's work), and each rank runs its wakes as one forest.

Results stay on their rank; ``gather`` (an all-gather over the process group, NCCL between GPUs) reassembles the full
array in the original target order when a caller needs it there.
"""
import numpy as np
import torch

_BITS = 21


def _spread(v):
    """Spread the low 21 bits of v (uint64) to every third bit."""
    v = v & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def morton_order(points):
    """Stable order of points by the 63-bit Morton key of their cell in the points' bounding cube."""
    points = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    if len(points) == 0:
        return np.zeros(0, dtype=np.int64)
    lo = points.min(axis=0)
    extent = float((points.max(axis=0) - lo).max())
    scale = ((1 << _BITS) - 1) / extent if extent > 0 else 0.0
    q = np.clip(np.floor((points - lo) * scale), 0, (1 << _BITS) - 1).astype(np.uint64)
    keys = (_spread(q[:, 0]) << np.uint64(2)) | (_spread(q[:, 1]) << np.uint64(1)) | _spread(q[:, 2])
    return np.argsort(keys, kind="stable").astype(np.int64)


def target_shards(points, world):
    """Per-rank index arrays: contiguous ranges of the Morton order, sizes differing by at most one."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    order = morton_order(points)
    bounds = np.linspace(0, len(order), world + 1).round().astype(np.int64)
    return [order[bounds[r]:bounds[r + 1]] for r in range(world)]


def wake_cost(segments, targets):
    return float(segments) * np.sqrt(max(float(targets), 1.0)) + float(targets)


def wake_shards(sizes, world):
    """Assign wakes given as (segments, targets) pairs to ranks: largest cost first, to the least-loaded rank (lowest
    rank on ties).  Returns per-rank lists of wake indices, each in increasing order, and the per-rank loads."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    costs = np.array([wake_cost(s, t) for s, t in sizes])
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for w in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = int(np.argmin(load))
        owner[w] = r
        load[r] += costs[w]
    return [sorted(np.flatnonzero(owner == r).tolist()) for r in range(world)], load


def gather(local, index, total, group=None):
    """All-gather each rank's rows `local` [k, ...] of targets `index` [k] into a [total, ...] tensor in target order.

    Ranks may hold different row counts; every rank makes the same two collective calls."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = local.device
    count = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(count) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    counts = [int(c.item()) for c in counts]
    width = max(counts) if counts else 0
    tail = tuple(local.shape[1:])
    pad = torch.zeros((width,) + tail, dtype=local.dtype, device=dev)
    pad[:local.shape[0]] = local
    idx = torch.full((width,), -1, dtype=torch.int64, device=dev)
    idx[:local.shape[0]] = torch.as_tensor(index, dtype=torch.int64, device=dev)
    rows = [torch.empty_like(pad) for _ in range(world)]
    idxs = [torch.empty_like(idx) for _ in range(world)]
    dist.all_gather(rows, pad, group=group)
    dist.all_gather(idxs, idx, group=group)
    out = torch.empty((total,) + tail, dtype=local.dtype, device=dev)
    for r in range(world):
        k = counts[r]
        out[idxs[r][:k]] = rows[r][:k]
    return out


def sharded_tree_sum(sources, points, rank, world, model, precision="mixed", theta=0.04, order=2, leaf_size=32,
                     block=128, singularity="raise", kind="morton"):
    """This rank's share of one wake: (target indices, velocity [k,3], flags [k]) with the tree built from all the
    (replicated) segments and evaluated at this rank's Morton range of targets."""
    from . import engine
    shard = target_shards(points, world)[rank]
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)[shard]
    tgt = engine.Targets(pts, None, sources.device)
    u, flags, _ = engine.tree_sum(sources, tgt, model, singularity, precision, block, 3.0, theta, order, leaf_size,
                                  3.0, kind, far_counts=False)
    return shard, u, flags
