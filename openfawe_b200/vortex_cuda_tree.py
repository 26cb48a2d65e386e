"""Drop-in for the reference's GPU tree backend ``openfawe.aero.vortex_cuda_tree`` (src/openfawe/aero/vortex_cuda_tree.py).

Same public names and call signature: ``Statistics`` and ``cuda_tree_sum(points, starts, directions, lengths, gamma,
radius, model, csr, singularity, tree, settings, *, targets_per_launch=None, stack_size=512, block=None) ->
(out, any_flag)`` (vortex_cuda_tree.py:439-595).  Everything runs on the device in libbs_b200:

* the tree: by default the reference's median-split tree (vortex_tree.build_tree), element for element, built on the
  GPU; with ``settings.tree == 'morton'`` this library's Morton-key tree;
* node centres, bounding radii, largest cores, moments and contractions in FP64 (vortex_tree.node_moments);
* the traversal of vortex_tree.tree_velocity with the FP64 acceptance test of the reference's GPU kernels, so the
  accepted nodes are those of the CPU tree code; ``fp64`` evaluates pairs and expansions in FP64, ``mixed``/``fp32``
  in FP32 on two-float coordinates with FP64 re-evaluation near segments (no target goes to the CPU, whatever
  ``settings.suspect`` says).

Errors as in the reference: ValueError for unsupported core models, theta >= 1, fp64 with suspect='gpu64' and a missing
device; RuntimeError for a traversal stack overflow.  ``targets_per_launch`` is accepted and ignored; ``stack_size``
caps the traversal stack (its maximum here is 128 entries per warp, enough for trees of depth 127).
"""
import time

import numpy as np

from . import vortex_cuda as VC

STACK = 512
TARGETS_PER_LAUNCH = 65536
PRECISIONS = ("fp64", "mixed", "fp32")
SUPPORTED_MODELS = (0, 1, 2)  # NONE, RANKINE, LAMB_OSEEN (vortex_tree.py:46)
DEVICE_STACK = 128


# Options set by ``configure`` (or ``openfawe_b200.install(...)``) for callers that pass the reference's own settings
# objects, which cannot express them: its TreeSettings refuses orders above 2 and its CudaSettings has no tree field
# (vortex.py:30-116).  Each one changes the approximation the caller asked for, and ``Statistics.last['effective']``
# records what a call ran.
OPTIONS = {}
_OPTION_NAMES = ("tree", "order", "theta", "leaf_size")


def configure(tree=None, order=None, theta=None, leaf_size=None):
    """Set (or, with no arguments, clear) the options every later ``cuda_tree_sum`` call applies.

    * ``tree``: 'median' or 'morton', for calls whose settings have no ``tree`` field (an explicit field wins);
    * ``order``: expansion order 0-5 in place of ``TreeSettings.order`` (the ``order=`` keyword of a call wins);
    * ``theta``: the opening ratio in place of ``TreeSettings.theta``: a number, a dict {caller's theta: theta}
      (thetas not in it are kept), or a callable of the caller's theta;
    * ``leaf_size``: in place of ``TreeSettings.leaf_size``.
    Returns the previous options."""
    if tree is not None and tree not in ("median", "morton"):
        raise ValueError("tree must be 'median' or 'morton'")
    if order is not None and order not in (0, 1, 2, 3, 4, 5):
        raise ValueError("tree order must be 0, 1, 2, 3, 4 or 5")
    if leaf_size is not None and (isinstance(leaf_size, bool) or int(leaf_size) < 1):
        raise ValueError("leaf size must be a positive integer")
    if theta is not None and not (callable(theta) or isinstance(theta, dict)) and not 0 < float(theta) < 1:
        raise ValueError("tree theta must lie strictly between 0 and 1")
    previous = dict(OPTIONS)
    OPTIONS.clear()
    OPTIONS.update({k: v for k, v in zip(_OPTION_NAMES, (tree, order, theta, leaf_size)) if v is not None})
    return previous


def effective(tree, settings, order=None):
    """(kind, order, theta, leaf_size) that a call with these settings runs under the configured options."""
    kind = getattr(settings, "tree", None) or OPTIONS.get("tree", "median")
    expansion = int(order if order is not None else OPTIONS.get("order", tree.order))
    theta = float(tree.theta)
    mapped = OPTIONS.get("theta")
    if callable(mapped):
        theta = float(mapped(theta))
    elif isinstance(mapped, dict):
        theta = float(mapped.get(theta, theta))
    elif mapped is not None:
        theta = float(mapped)
    leaf = int(OPTIONS.get("leaf_size", tree.leaf_size))
    return kind, expansion, theta, leaf


class Statistics:
    last = {}
    last_far_counts = None
    totals = dict(calls=0, suspect=0, launches=0)

    @classmethod
    def reset_totals(cls):
        cls.totals = dict(calls=0, suspect=0, launches=0)


def cuda_tree_sum(points, starts, directions, lengths, gamma, radius, model, csr, singularity, tree, settings, *,
                  targets_per_launch=None, stack_size=STACK, block=None, order=None):
    """Return (velocity, any_flag) like ``vortex_tree.tree_sum`` for the same inputs, evaluated on the GPU.

    ``order`` (keyword, not in the reference) overrides ``tree.order``; 3, 4 and 5 select the third- to fifth-order
    far fields, which reach the accuracy of order 2 at larger opening angles.  Options set by ``configure`` apply to
    every call (see there)."""
    if not VC.available():
        raise ValueError(f"the cuda tree evaluation needs a CUDA device ({VC.probe_error()})")
    if int(model) not in SUPPORTED_MODELS and np.any(np.asarray(radius) > 0):
        raise ValueError("tree backend supports core models NONE, RANKINE and LAMB_OSEEN only")
    if tree.theta >= 1.0:
        raise ValueError("tree theta must be below one")
    kind, expansion, theta, leaf_size = effective(tree, settings, order)
    if not 0.0 < theta < 1.0:
        raise ValueError("tree theta must lie strictly between 0 and 1 (after the configured mapping)")
    precision = settings.precision
    gpu64 = getattr(settings, "suspect", "cpu") == "gpu64"
    if gpu64 and precision == "fp64":
        raise ValueError("suspect='gpu64' is for the single precisions only")
    block = int(settings.block if block is None else block)
    if expansion not in (0, 1, 2, 3, 4, 5):
        raise ValueError("tree order must be 0, 1, 2, 3, 4 or 5")
    _, _, near = VC._check_settings(settings)
    points = np.ascontiguousarray(points, dtype=np.float64)
    n, m = len(points), len(starts)
    if n == 0 or m == 0:
        Statistics.last = dict(points=n, segments=m, launches=0, suspect=0)
        if gpu64:
            Statistics.last.update(suspect_mode="gpu64", suspect_targets=0, suspect_pairs=0)
        return np.zeros((n, 3)), False
    import torch
    from . import _lib, engine
    device = torch.cuda.current_device()
    limit = int(stack_size) if 0 < int(stack_size) < DEVICE_STACK else 0
    try:
        if any(isinstance(x, torch.Tensor) for x in (starts, directions, lengths, gamma, radius)):
            # device-resident inputs: build, moments and evaluation in one library call, then the three results
            tick = time.perf_counter()
            sources = engine.Sources(starts, directions, lengths, gamma, radius, device)
            targets = engine.Targets(points, csr, device)
            upload_s = time.perf_counter() - tick
            tick = time.perf_counter()
            d_out, d_flags, d_far = engine.tree_sum(sources, targets, int(model), singularity, precision, block,
                                                    near, theta, expansion, leaf_size, tree.core_clearance, kind,
                                                    stack_limit=limit)
            total_s = time.perf_counter() - tick
            tick = time.perf_counter()
            out, flags, far = engine.to_host_many((d_out, d_flags, d_far), ((n, 3), (n,), (n,)),
                                                  (np.float64, np.int8, np.int64))
            download_s = time.perf_counter() - tick
            stats = engine.last_stats(device)
        else:
            # host arrays: one library call from the host arrays to the host results (uploads overlap the build)
            tick = time.perf_counter()
            out, flags, far = engine.tree_sum_host(points, starts, directions, lengths, gamma, radius, csr,
                                                   int(model), singularity, precision, block, near, theta,
                                                   expansion, leaf_size, tree.core_clearance, kind, limit, device)
            stats = engine.last_stats(device)
            upload_s, download_s = 1e-3 * stats["upload_ms"], 1e-3 * stats["download_ms"]
            total_s = time.perf_counter() - tick - upload_s - download_s
    except _lib.StackOverflow as error:
        raise RuntimeError(f"tree traversal stack overflow on the GPU (depth {min(int(stack_size), DEVICE_STACK)})") \
            from error
    build_s = 1e-3 * (stats["build_ms"] + stats["moments_ms"])
    evaluate_s = max(0.0, total_s - build_s)
    Statistics.last = dict(points=n, segments=m, nodes=int(stats["nodes"]), precision=precision, launches=1,
                           targets_per_launch=n, longest_launch_s=stats["evaluate_ms"] * 1e-3, suspect=0,
                           mean_far_nodes=float(far.mean()), build_s=build_s, moments_s=0.0, upload_s=upload_s,
                           evaluate_s=evaluate_s, download_s=download_s, recompute_s=0.0, tree=kind,
                           build_ms=stats["build_ms"], moments_ms=stats["moments_ms"],
                           evaluate_ms=stats["evaluate_ms"], near_pairs=int(stats["near_pairs"]),
                           far_evaluations=int(stats["far_evaluations"]), fp64_pairs=int(stats["fp64_pairs"]),
                           visits=int(stats["visits"]),
                           effective=dict(tree=kind, order=expansion, theta=theta, leaf_size=leaf_size),
                           **({"moments": "gpu"} if getattr(settings, "moments", "cpu") == "gpu" else {}),
                           **({"build": "gpu"} if getattr(settings, "build", "cpu") == "gpu" else {}))
    if gpu64:
        Statistics.last.update(suspect_mode="gpu64", suspect_targets=0, suspect_pairs=int(stats["fp64_pairs"]))
    Statistics.last_far_counts = far
    Statistics.totals["calls"] += 1
    Statistics.totals["launches"] += 1
    return out, bool(np.any(flags))
