"""Batched evaluation of many independent wakes of uneven sizes in one persistent launch.

A ``WakeBatch`` concatenates the segments and targets of many wakes of uneven sizes (a wind-speed sweep, several time
steps), builds one forest on the device (``bs_forest_build``: one key sort and one radix tree whose upper splits fall
on wake boundaries) and evaluates every wake at its own targets with one traversal launch and one persistent list
kernel (``bs_forest_eval``), optionally captured as a CUDA graph and replayed (``bs_forest_graph``).  The reference
evaluates one wake per call; ``sequential`` times that pattern on the same wakes.

``autotune`` is the project's tuner of the launch shapes: it times candidate leaf sizes and traversal block sizes on
the batch itself with CUDA events and keeps the fastest per size class of batch.

Control points: the reference's VSM free wake also sums every wake exactly at its wing's control and load points
(vsm_wake.history_vsm_induction, src/openfawe/aero/vsm_wake.py:255-300).  ``WakeBatch(cases, control=[points of wake
0, ...])`` appends those points to each wake's targets, marked exact (no far node is accepted for them), so both
sums of every wake run in the one traversal and persistent list launch (and graph); ``split_control`` returns them.
"""
import numpy as np
import torch

from . import engine

_TUNED = {}


class WakeBatch:
    """Wakes given as backend-argument dicts (``wakes.rotor_sheet`` and friends: points, starts, directions, lengths,
    gamma, radius, model); all wakes share the core model."""

    def __init__(self, cases, device=0, leaf_size=32, control=None):
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        models = {int(c["model"]) for c in cases}
        if len(models) != 1:
            raise ValueError("all wakes of a batch must use one core model")
        self.model = models.pop()
        if control is not None and len(control) != len(cases):
            raise ValueError("control: one point array per wake (or None)")
        ctrl = [np.zeros((0, 3)) if control is None or control[w] is None
                else np.asarray(control[w], dtype=np.float64).reshape(-1, 3) for w in range(len(cases))]
        seg_counts = [len(c["starts"]) for c in cases]
        own_counts = [len(c["points"]) for c in cases]
        tgt_counts = [a + len(b) for a, b in zip(own_counts, ctrl)]
        self.wake_ptr = np.concatenate(([0], np.cumsum(seg_counts))).astype(np.int64)
        self.target_ptr = np.concatenate(([0], np.cumsum(tgt_counts))).astype(np.int64)
        self.own_counts = own_counts
        cat = lambda key: np.concatenate([c[key] for c in cases])  # noqa: E731
        self.sources = engine.Sources(cat("starts"), cat("directions"), cat("lengths"), cat("gamma"), cat("radius"),
                                      self.device)
        points = np.concatenate([np.concatenate((c["points"], q)) for c, q in zip(cases, ctrl)])
        self.exact = None
        if control is not None:
            self.exact = np.concatenate([np.concatenate((np.zeros(len(c["points"]), np.uint8),
                                                         np.ones(len(q), np.uint8))) for c, q in zip(cases, ctrl)])
        self.targets = engine.Targets(points, None, self.device)
        self.leaf_size = leaf_size
        self.order = 2
        self.forest = None
        self.graph = None

    @property
    def count(self):
        return len(self.wake_ptr) - 1

    def build(self, leaf_size=None, order=None):
        if leaf_size is not None:
            self.leaf_size = leaf_size
        if order is not None:
            self.order = order
        self.forest = engine.build_forest(self.sources, self.wake_ptr, self.leaf_size, self.order)
        self.graph = None
        return self.forest

    def evaluate(self, theta=0.04, order=2, precision="mixed", block=128, singularity="raise", near=3.0):
        """(velocity [n_total,3], flags, far counts) as device tensors; split with ``split``."""
        if self.forest is None:
            self.build()
        return engine.forest_eval(self.forest, self.targets, self.target_ptr, self.model, singularity, precision,
                                  block, near, theta, order, exact=self.exact)

    def capture(self, theta=0.04, order=2, precision="mixed", block=128, singularity="raise", near=3.0):
        """Capture the evaluation as a CUDA graph (``launch()`` replays it)."""
        if self.forest is None:
            self.build()
        self.graph = engine.Graph(self.forest, self.targets, self.target_ptr, self.model, singularity, precision, block,
                                  near, theta, order, exact=self.exact)
        return self.graph

    def split(self, array):
        """Per-wake views of a concatenated per-target array (each wake's own targets; control points left out)."""
        return [array[a:a + k] for a, k in zip(self.target_ptr[:-1], self.own_counts)]

    def split_control(self, array):
        """Per-wake views of the control points' rows of a concatenated per-target array."""
        return [array[a + k:b] for a, k, b in zip(self.target_ptr[:-1], self.own_counts, self.target_ptr[1:])]


def device_ms(fn, repeats=3):
    """Best CUDA-event time of `fn` over `repeats` calls after one warm-up call."""
    fn()
    torch.cuda.synchronize()
    best = np.inf
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def autotune(batch, theta=0.04, precision="mixed", leaves=(16, 32, 64), blocks=(64, 128), order=2):
    """Pick (leaf_size, block) for this batch's size class by timing build + evaluation; returns the choice and the
    table of timings.  Results are cached per (segments, targets, wakes) size class within the process."""
    key = (int(np.log2(max(1, batch.sources.m))), int(np.log2(max(1, batch.targets.n))), batch.count, theta, precision,
           order)
    if key in _TUNED:
        batch.build(_TUNED[key]["choice"][0], order)
        return _TUNED[key]
    table = {}
    for leaf in leaves:
        for block in blocks:
            table[(leaf, block)] = device_ms(
                lambda: (batch.build(leaf, order), batch.evaluate(theta, order, precision=precision, block=block)),
                repeats=2)
    choice = min(table, key=table.get)
    batch.build(choice[0], order)
    _TUNED[key] = dict(choice=choice, table={f"leaf{k[0]}_block{k[1]}": v for k, v in table.items()})
    return _TUNED[key]


def sequential(cases, device=0, theta=0.04, precision="mixed", leaf_size=32, block=128, kind="morton", order=2):
    """One tree_sum call per wake (the reference's pattern), inputs already on the device; per-wake CUDA-event ms."""
    dev = torch.device("cuda", device) if isinstance(device, int) else device
    data = [(engine.Sources(c["starts"], c["directions"], c["lengths"], c["gamma"], c["radius"], dev),
             engine.Targets(c["points"], None, dev), int(c["model"])) for c in cases]
    times, outs = [], []
    torch.cuda.synchronize()
    for src, tgt, model in data:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        u, _, _ = engine.tree_sum(src, tgt, model, "raise", precision, block, 3.0, theta, order, leaf_size, 3.0, kind,
                                  far_counts=False)
        e1.record()
        outs.append(u)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return np.array(times), outs
