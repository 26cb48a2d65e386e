"""Sharding of the induced-velocity sums over the GPUs of one node (one process per GPU).

The velocity at a target is a sum over segments, and every target is independent, so one wake splits two ways:

* by sources (the default for one wake): each rank takes a contiguous range of the segments' Morton order (spatially
  compact, so each rank's tree is a compact piece of the wake), builds its own tree over them and evaluates every
  target against it; one all-reduce (sum) of the [n, 3] FP64 partial velocities -- 494 KB at 20,570 targets, NCCL
  over NVLink between GPUs -- gives every rank the full result.  Build, moments and traversal all shrink with the
  rank count; only the far evaluations per target shrink more slowly (each rank still needs the far field of its piece
  at every target);
* by targets: the segments (and so the tree and its moments) are replicated on every rank, the targets are split into
  contiguous ranges of their Morton order of equal size; each rank evaluates its own range with no collective, and
  ``gather`` reassembles the full array when a caller needs it.  The build is not divided;
* a batch of wakes: wakes are assigned whole to ranks, largest first to the least-loaded rank (cost = segments x
  targets^(1/2) + targets, a stand-in for the tree's work), and each rank runs its wakes as one forest.

The orchestration (``sharded_sum``) takes the per-rank evaluation as a function, so the same code runs the library's
tree sum between GPUs and a CPU evaluation between gloo ranks in the tests.
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


def source_shards(starts, directions, lengths, world):
    """Per-rank segment index arrays: contiguous ranges of the Morton order of the segment midpoints, sizes differing
    by at most one."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    starts = np.asarray(starts, dtype=np.float64).reshape(-1, 3)
    mid = starts + 0.5 * np.asarray(directions, dtype=np.float64).reshape(-1, 3) * \
        np.asarray(lengths, dtype=np.float64).reshape(-1, 1)
    order = morton_order(mid)
    bounds = np.linspace(0, len(order), world + 1).round().astype(np.int64)
    return [np.sort(order[bounds[r]:bounds[r + 1]]) for r in range(world)]


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


def sharded_sum(evaluate, points, segments, rank, world, mode="sources", group=None):
    """One wake's induced velocity at every target, shared over the ranks of `group`.

    ``segments`` = (starts, directions, lengths, gamma, radius) host arrays; ``evaluate(points, starts, directions,
    lengths, gamma, radius)`` returns (velocity [k, 3] float64 tensor, flags [k] int8 tensor) on this rank's device.
    ``mode='sources'``: this rank evaluates every target against its Morton range of segments, then the partial
    velocities are summed (all-reduce) and the flags combined (maximum) over the ranks; ``mode='targets'``: this rank
    evaluates its Morton range of targets against every segment and the rows are all-gathered.  Every rank makes the
    same collective calls in the same order.  Returns (velocity [n, 3], flags [n]) in target order on every rank."""
    import torch.distributed as dist
    points = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    starts, directions, lengths, gamma, radius = (np.asarray(a, dtype=np.float64) for a in segments)
    starts, directions = starts.reshape(-1, 3), directions.reshape(-1, 3)
    if mode == "sources":
        mine = source_shards(starts, directions, lengths, world)[rank]
        u, flags = evaluate(points, starts[mine], directions[mine], lengths[mine], gamma[mine], radius[mine])
        u = u.to(torch.float64).contiguous()
        f = flags.to(torch.int32).contiguous()
        dist.all_reduce(u, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(f, op=dist.ReduceOp.MAX, group=group)
        return u, f.to(torch.int8)
    if mode == "targets":
        mine = target_shards(points, world)[rank]
        u, flags = evaluate(points[mine], starts, directions, lengths, gamma, radius)
        full_u = gather(u.to(torch.float64), mine, len(points), group)
        full_f = gather(flags.to(torch.int32).reshape(-1, 1), mine, len(points), group).reshape(-1)
        return full_u, full_f.to(torch.int8)
    raise ValueError("mode must be 'sources' or 'targets'")


def tree_evaluator(model, device, precision="mixed", theta=0.215, order=5, leaf_size=384, block=128,
                   singularity="raise", kind="morton"):
    """``evaluate`` for ``sharded_sum``: the library's tree sum (build, moments, traversal) on `device`."""
    from . import engine

    def evaluate(points, starts, directions, lengths, gamma, radius):
        src = engine.Sources(starts, directions, lengths, gamma, radius, device)
        tgt = engine.Targets(points, None, device)
        u, flags, _ = engine.tree_sum(src, tgt, model, singularity, precision, block, 3.0, theta, order, leaf_size,
                                      3.0, kind, far_counts=False)
        return u, flags
    return evaluate


def sharded_tree_sum(sources, points, rank, world, model, precision="mixed", theta=0.04, order=2, leaf_size=32,
                     block=128, singularity="raise", kind="morton"):
    """This rank's share of one wake split by targets: (target indices, velocity [k,3], flags [k]) with the tree built
    from all the (replicated, device-resident) segments and evaluated at this rank's Morton range of targets; no
    collective."""
    from . import engine
    shard = target_shards(points, world)[rank]
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)[shard]
    tgt = engine.Targets(pts, None, sources.device)
    u, flags, _ = engine.tree_sum(sources, tgt, model, singularity, precision, block, 3.0, theta, order, leaf_size,
                                  3.0, kind, far_counts=False)
    return shard, u, flags
