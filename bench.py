#!/usr/bin/env python
"""Benchmark of the free-wake induced-velocity hot path on B200.

Workload: a 3,744-row rotor-ring + wing-sheet wake (819,890 straight segments, Lamb-Oseen core 0.05 m, circulation
~ U(0, 8)) induced at 20,570 targets; seeded synthetic data of the shapes of the reference's README wakes.  One step
is one call of the mixed-precision tree path (Morton-key tree build + FP64 moments + traversal with FP32 far field and
pairs, FP64 near field and per-target sums) with inputs resident in HBM.  Reported beside it: the plain FP64 GPU
direct sum on the same inputs (the reference's 'cuda' fp64 backend's job), the relative L2 and max error of the
tree against that FP64 direct sum, the end-to-end time of the drop-in ``cuda_tree_sum`` from host NumPy arrays, and
the reference's CPU tree code (its CPU restatement in oracle/) on the host's cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
import argparse
import ctypes
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "ms/call at 102k-820k segs, mixed vs FP64 at <=1e-6 rel err; adjoint/fwd ratio"
ROWS, TARGETS, SEED = 3744, 20570, 3744
THETA, ORDER, LEAF, CLEARANCE = 0.215, 5, 384, 3.0
# The reference's CPU tree code has orders 0-2; on this workload it reaches the same <= 1e-6 relative L2 error against
# the FP64 direct sum at order 2 and theta 0.04 (7.5e-7), which is the setting its baseline is timed at.
REF_THETA, REF_ORDER, REF_LEAF = 0.04, 2, 32
W_PAIR, W_VISIT = 62.0, 12.0            # algorithmic flops per near pair and per visited node
LIST_TRAFFIC = 8.57e6                   # DRAM bytes read + written by one near-leaf kernel launch of the default
                                        # step (ncu dram__bytes_read.sum + dram__bytes_write.sum; records L2-resident)
# per far evaluation of order p (3: 180 + 170 for the third term, 4: 350 + 300 for the fourth)
W_FAR = {0: 40.0, 1: 100.0, 2: 180.0, 3: 350.0, 4: 650.0, 5: 1100.0}
L2_FLUSH_BYTES = 512 << 20  # larger than the 126 MB L2
GOLDEN = os.path.join(HERE, "tests", "golden")
ACCURACY_SAMPLE = 256  # targets at which the reference arm's CPU tree is checked against the oracle's FP64 direct sum
# The reference's published figures for the 468-row self-test sheet at theta 0.2, order 2, leaf 32 (README.md:88;
# RTX 4090 D and 22 CPU threads, median of five calls), seconds.
README_468 = {"cpu_1_thread_s": 2.07, "cpu_22_threads_s": 0.16, "gpu_double_s": 0.14, "gpu_mixed_s": 0.07,
              "hardware": "NVIDIA RTX 4090 D, 22 CPU threads"}


@dataclass(frozen=True)
class CallerTreeSettings:
    """The reference's TreeSettings as a caller holds it (vortex.py:30-55): these fields and no others."""
    theta: float = 0.5
    order: int = 2
    leaf_size: int = 32
    core_clearance: float = 3.0


@dataclass(frozen=True)
class CallerCudaSettings:
    """The reference's CudaSettings as a caller holds it (vortex.py:58-116): no tree field."""
    precision: str = "mixed"
    block: int = 128
    suspect: str = "cpu"
    control: str = "cpu"
    moments: str = "cpu"
    build: str = "cpu"
    rings: str = "cpu"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=("b200", "reference"))
    p.add_argument("--rows", type=int, default=ROWS)
    p.add_argument("--theta", type=float, default=THETA)
    p.add_argument("--leaf", type=int, default=LEAF)
    p.add_argument("--order", type=int, default=ORDER, choices=(0, 1, 2, 3, 4, 5))
    p.add_argument("--kind", default="morton", choices=("morton", "median"))
    p.add_argument("--no-extras", action="store_true",
                   help="skip the batched-wakes, adjoint, C1, C2 and default-path measurements")
    p.add_argument("--only", default=None, choices=("tree", "direct-fp64", "direct-mixed", "adjoint",
                                                    "tree-adjoint"),
                   help="run one call kind alone, warmup + steps times, and print its counters (for profiler runs)")
    p.add_argument("--tree-only", action="store_const", const="tree", dest="only", help="the same as --only tree")
    p.add_argument("--reference-gpu-leg", action="store_true", help=argparse.SUPPRESS)
    return p.parse_args()


REF_INSTALL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "baseline", "_ref")


def reference_gpu_leg(args):
    """(Subprocess) the reference's own numba.cuda tree code (vortex_cuda_tree.cuda_tree_sum with the GPU build and
    moments, vortex.py:58-116), installed under baseline/_ref, on the bench wake from host arrays, as its callers use
    it: its production setting (theta 0.2, order 2, leaf 32; mixed with the GPU FP64 suspect pairs, and FP64) and
    its equal-accuracy setting (theta 0.04); the first call of each compiles its kernels, the next three are timed."""
    sys.path.insert(0, REF_INSTALL)
    import torch
    from openfawe.aero import vortex as RV, vortex_cuda_tree as RVCT
    from openfawe_b200 import engine
    case = workload(args.rows)
    segments = [case[k] for k in ("starts", "directions", "lengths", "gamma", "radius")]
    n = len(case["points"])
    csr = (np.zeros(n + 1, dtype=np.int64), np.zeros(0, dtype=np.int64))
    device = torch.device("cuda", 0)
    src = engine.Sources(*segments, device)
    tgt = engine.Targets(case["points"], None, device)
    direct = engine.direct(src, tgt, case["model"], "raise", "fp64")[0].cpu().numpy()
    out = {"implementation": "the reference's numba.cuda cuda_tree_sum (baseline/_ref), build='gpu', moments='gpu'",
           "workload": config(case, args)["workload"]}
    for theta, precision, suspect in ((0.2, "mixed", "gpu64"), (0.2, "fp64", "cpu"), (0.04, "mixed", "gpu64")):
        tree = RV.TreeSettings(theta=theta, order=2, leaf_size=32, core_clearance=CLEARANCE)
        cuda = RV.CudaSettings(precision, 128, suspect, moments="gpu", build="gpu")
        times, u = [], None
        for rep in range(4):
            torch.cuda.synchronize()
            tick = time.perf_counter()
            u, _ = RVCT.cuda_tree_sum(case["points"], *segments, case["model"], csr, "raise", tree, cuda)
            times.append((time.perf_counter() - tick) * 1e3)
        out[f"theta_{theta}_{precision}"] = {
            "ms_per_call": float(np.median(times[1:])), "first_call_ms": times[0],
            "rel_l2_vs_fp64_direct": float(np.linalg.norm(u - direct) / np.linalg.norm(direct))}
    print(json.dumps(out), flush=True)
    return 0


def reference_gpu_measure():
    """The reference's own GPU tree code on this GPU (reference_gpu_leg, in a process of its own so that nothing of
    this library's drop-in touches its modules), when it is installed under baseline/_ref."""
    if not os.path.isdir(os.path.join(REF_INSTALL, "openfawe")):
        return {"unavailable": "the reference is not installed under baseline/_ref"}
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--reference-gpu-leg"], capture_output=True,
                           text=True, timeout=900)
        return json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else {
            "unavailable": f"exit {r.returncode}: {r.stderr.strip().splitlines()[-1] if r.stderr.strip() else ''}"}
    except Exception as exc:  # a failed leg is reported, not fatal
        return {"unavailable": repr(exc)}


def workload(rows):
    from openfawe_b200 import wakes
    return wakes.rotor_sheet(rows, seed=SEED, targets=TARGETS)


def config(case, args, extra=None):
    c = {"workload": f"rotor-sheet wake {args.rows} rows, {len(case['starts'])} segments x {len(case['points'])} "
                     f"targets, Lamb-Oseen rc 0.05 m",
         "segments": len(case["starts"]), "targets": len(case["points"]), "theta": args.theta, "order": args.order,
         "leaf_size": args.leaf, "tree": args.kind, "precision": "mixed", "l2": "flushed between timed steps (512 MB write)",
         "parallelism": ("one GPU" if args.gpus <= 1 else
                         f"one call shared by segments over {args.gpus} GPUs (Morton ranges, all-reduce of the result)")}
    if extra:
        c.update(extra)
    return c


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock, max clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        rows = [line.split(",") for line in self.file.read().strip().splitlines() if line.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = [name for k, name in enumerate(names) if any(r[5 + k].strip() == "Active" for r in rows)]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(path, encoding="utf-8") as f:
            return json.load(f)
    except OSError:
        return {}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def no_exclusions(n):
    return np.zeros(n + 1, dtype=np.int64), np.zeros(0, dtype=np.int64)


def cpu_tree_call(case, theta, order=REF_ORDER, leaf=REF_LEAF, points=None):
    """One full call of the reference's CPU tree code (vortex_tree.tree_sum, restated in oracle/) on every host core:
    median-split build, moments, contractions and the traversal of every target.  Returns (seconds, velocity)."""
    from oracle import oracle as O
    from openfawe_b200 import wakes
    args = wakes.backend_args(case)
    if points is not None:
        args = (points, *args[1:])
    tick = time.perf_counter()
    u, _ = O.tree_sum(*args, no_exclusions(len(args[0])), "raise", theta, order, leaf, CLEARANCE, "median")
    return time.perf_counter() - tick, u


def sample_accuracy(case, u):
    """Relative L2 and max error of `u` against the oracle's FP64 direct sum at ACCURACY_SAMPLE evenly spaced targets."""
    from oracle import oracle as O
    from openfawe_b200 import wakes
    n = len(case["points"])
    pick = np.linspace(0, n - 1, min(ACCURACY_SAMPLE, n)).astype(np.int64)
    args = wakes.backend_args(case)
    ref, _ = O.direct_sum(case["points"][pick], *args[1:], no_exclusions(len(pick)), "raise")
    err = np.linalg.norm(u[pick] - ref, axis=1)
    return {"rel_l2": float(np.linalg.norm(u[pick] - ref) / np.linalg.norm(ref)),
            "max_err_over_max_speed": float(err.max() / np.linalg.norm(ref, axis=1).max()),
            "sample": f"{len(pick)} evenly spaced targets against the oracle's FP64 direct sum"}


def errors(u, ref):
    err = np.linalg.norm(u - ref, axis=1)
    return {"rel_l2": float(np.linalg.norm(u - ref) / np.linalg.norm(ref)),
            "max_err_over_max_speed": float(err.max() / np.linalg.norm(ref, axis=1).max())}


def cpu_baseline(case, direct_host=None):
    """The reference's CPU tree code (oracle port) timed on the host's cores: one full call at its setting for the same
    <= 1e-6 accuracy (order 2, theta 0.04), every target."""
    seconds, u = cpu_tree_call(case, REF_THETA)
    base = {"value": 1e3 * seconds, "unit": "ms/call", "cores": host_cores(), "kind": "port",
            "sample": f"one full call, all {len(case['points'])} targets: median-split build, moments and traversal at "
                      f"theta {REF_THETA}, order {REF_ORDER}, leaf {REF_LEAF} (the reference's orders stop at 2; "
                      f"this is its setting for the same <= 1e-6 error)"}
    if direct_host is not None:
        base["accuracy_vs_fp64_direct"] = errors(u, direct_host)
    return base


def reference_arm(args):
    """The reference's CPU tree code (its restatement in oracle/, C with OpenMP on every host core) on the same wake
    and metric: each step is one full call (build, moments, traversal of every target), timed whole."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    case = workload(args.rows)
    times, u = [], None
    for step in range(args.warmup + args.steps):
        seconds, u = cpu_tree_call(case, REF_THETA)
        if step >= args.warmup:
            times.append(1e3 * seconds)
    value = statistics.median(times)
    rows = {}
    for theta, label in ((0.5, "reference default"), (0.2, "production setting")):
        runs = [cpu_tree_call(case, theta) for _ in range(3)]
        rows[f"theta_{theta}"] = {"setting": label, "ms_per_call": 1e3 * statistics.median(r[0] for r in runs),
                                  "accuracy": sample_accuracy(case, runs[-1][1])}
    base = {"value": value, "unit": "ms/call", "cores": host_cores(), "kind": "port",
            "sample": f"full calls on all {len(case['points'])} targets, median of {args.steps} after {args.warmup} "
                      f"warm-up calls; theta {REF_THETA}, order {REF_ORDER}, leaf {REF_LEAF}, median-split tree",
            "accuracy": sample_accuracy(case, u), "other_settings": rows}
    line = {"metric": METRIC, "value": value, "unit": "ms/call", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(case, args, {"precision": "fp64 (CPU tree code)", "tree": "median", "theta": REF_THETA,
                                          "order": REF_ORDER, "leaf_size": REF_LEAF,
                                          "l2": "not applicable (CPU)"}),
            "cpu_baseline": base, "e2e": {"value": value, "unit": "ms/call", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _event_ms(fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def batch_measure(device, theta, order=ORDER):
    """48 rotor-sheet wakes of 5k-410k segments (a wind sweep) in one forest: autotuned build + evaluation, the
    evaluation alone, its CUDA-graph replay, and the same wakes one tree_sum call each (the reference's pattern)."""
    import torch
    from openfawe_b200 import batch, wakes
    cases = wakes.wake_batch(48, seed=48)
    b = batch.WakeBatch(cases, device)
    b.order = order
    tuned = batch.autotune(b, theta=theta, leaves=(64, 128, 256, 384), blocks=(64, 128), order=order)
    leaf, block = tuned["choice"]
    total = min(_event_ms(lambda: (b.build(leaf), b.evaluate(theta, order, block=block))) for _ in range(3))
    evaluate = min(_event_ms(lambda: b.evaluate(theta, order, block=block)) for _ in range(3))
    graph = b.capture(theta, order, block=block)
    graph.launch()
    torch.cuda.synchronize()
    replay = min(_event_ms(graph.launch) for _ in range(3))
    batch.sequential(cases[:4], device, theta=theta, leaf_size=leaf, block=block, order=order)   # warm the pool
    seq = min((batch.sequential(cases, device, theta=theta, leaf_size=leaf, block=block, order=order)[0]
               for _ in range(2)), key=lambda t: t.sum())
    # with each wake's 64-panel wing control points summed exactly in the same launch (the VSM induction), against
    # the reference's pattern of one tree call and one exact control-point call per wake
    from openfawe_b200 import engine
    control = [wakes.ring_wing(64)["points"] for _ in cases]
    bc = batch.WakeBatch(cases, device, leaf_size=leaf, control=control)
    bc.build(leaf, order)
    with_control = min(_event_ms(lambda: (bc.build(leaf, order), bc.evaluate(theta, order, block=block)))
                       for _ in range(3))
    gc = bc.capture(theta, order, block=block)
    gc.launch()
    torch.cuda.synchronize()
    replay_control = min(_event_ms(gc.launch) for _ in range(3))
    per_wake = []
    for c, q in zip(cases, control):
        src = engine.Sources(c["starts"], c["directions"], c["lengths"], c["gamma"], c["radius"], device)
        tgt, ctl = engine.Targets(c["points"], None, device), engine.Targets(q, None, device)
        run = lambda: (engine.tree_sum(src, tgt, c["model"], "raise", "mixed", block, 3.0, theta, order, leaf,  # noqa
                                       CLEARANCE, "morton", far_counts=False),
                       engine.direct(src, ctl, c["model"], "raise", "mixed"))
        run()
        per_wake.append(min(_event_ms(run) for _ in range(2)))
    per_wake = np.asarray(per_wake)
    return {"wakes": len(cases), "segments": int(b.sources.m), "targets": int(b.targets.n),
            "segments_per_wake": [int(min(len(c["starts"]) for c in cases)), int(max(len(c["starts"]) for c in cases))],
            "autotune": {"leaf_size": leaf, "block": block, "table_ms": tuned["table"]},
            "batched_total_ms": total, "batched_eval_ms": evaluate, "graph_replay_ms": replay,
            "sequential_total_ms": float(seq.sum()), "sequential_p50_ms": float(np.percentile(seq, 50)),
            "sequential_p99_ms": float(np.percentile(seq, 99)),
            "batched_per_wake_latency_ms": {"p50": total, "p99": total,
                                            "note": "every wake's result is ready when the one launch ends"},
            "batched_per_wake_mean_ms": total / len(cases), "speedup_vs_sequential": float(seq.sum()) / total,
            "with_control_points": {"control_points_per_wake": 64, "batched_total_ms": with_control,
                                    "graph_replay_ms": replay_control,
                                    "sequential_total_ms": float(per_wake.sum()),
                                    "sequential_p50_ms": float(np.percentile(per_wake, 50)),
                                    "sequential_p99_ms": float(np.percentile(per_wake, 99)),
                                    "speedup_vs_sequential": float(per_wake.sum()) / with_control,
                                    "sequential_call": "per wake: tree_sum of its own targets, then the exact "
                                                       "direct sum at its control points"}}


def adjoint_measure(device, theta, bench_case=None):
    """The hand-written adjoints (grads w.r.t. targets, both endpoints and circulations) against the forwards they
    differentiate: on the 468-row rotor sheet (C5) the exact FP64 adjoint against the FP64 direct sum, and the tree
    adjoint against the mixed fifth-order tree forward (with its error against the exact gradient); on the bench wake
    the tree adjoint against the bench's tree forward."""
    import torch
    from openfawe_b200 import adjoint, engine, wakes

    def setup(case):
        ends = case["nodes"][case["edges"][:, 1]]
        pts = torch.as_tensor(case["points"], device=device)
        a = torch.as_tensor(case["starts"], device=device)
        bb = torch.as_tensor(ends, device=device)
        gam = torch.as_tensor(case["gamma"], device=device)
        rad = torch.as_tensor(case["radius"], device=device)
        rng = np.random.default_rng(5)
        w = torch.as_tensor(rng.standard_normal((len(case["points"]), 3)).astype(np.float32).astype(np.float64),
                            device=device)
        src = engine.Sources(case["starts"], case["directions"], case["lengths"], case["gamma"], case["radius"],
                             device)
        tgt = engine.Targets(case["points"], None, device)
        return pts, a, bb, gam, rad, w, src, tgt

    case = wakes.rotor_sheet(468, seed=468, targets=20570)
    pts, a, bb, gam, rad, w, src, tgt = setup(case)
    model = case["model"]
    run_adj = lambda: adjoint.adjoint_direct(pts, a, bb, gam, rad, model, w)  # noqa: E731
    run_direct = lambda: engine.direct(src, tgt, model, "raise", "fp64")  # noqa: E731
    run_tree = lambda: engine.tree_sum(src, tgt, model, "raise", "mixed", 128, 3.0, theta, ORDER, LEAF,  # noqa: E731
                                       CLEARANCE, "morton", far_counts=False)
    run_tree_adj = lambda: adjoint.adjoint_tree(pts, a, bb, gam, rad, model, w, precision="mixed",  # noqa: E731
                                                theta=theta, order=ORDER, leaf_size=LEAF, kind="morton")
    for fn in (run_adj, run_direct, run_tree, run_tree_adj):
        fn()
    torch.cuda.synchronize()
    adj = min(_event_ms(run_adj) for _ in range(3))
    fwd = min(_event_ms(run_direct) for _ in range(3))
    tree = min(_event_ms(run_tree) for _ in range(5))
    tree_adj = min(_event_ms(run_tree_adj) for _ in range(5))
    stats = engine.last_stats(device)
    exact = [t.cpu().numpy() for t in run_adj()]
    approx = [t.cpu().numpy() for t in run_tree_adj()]
    err = {name: float(np.linalg.norm(u - v) / np.linalg.norm(v))
           for name, u, v in zip(("points", "starts", "ends", "gamma"), approx, exact)}
    out = {"workload": f"rotor-sheet wake 468 rows, {src.m} segments x {tgt.n} targets, cotangent N(0,1) seed 5",
           "adjoint_ms": adj, "fp64_direct_forward_ms": fwd, "mixed_tree_forward_ms": tree,
           "ratio_to_fp64_direct": adj / fwd, "ratio_to_tree_forward": adj / tree,
           "tree_adjoint": {"ms": tree_adj, "ratio_to_tree_forward": tree_adj / tree,
                            "stages_ms": {"build_walk_transpose": stats["build_ms"], "near_pairs": stats["walk_ms"],
                                          "far_entries": stats["list_ms"],
                                          "pushdown_segment_moments": stats["moments_ms"]},
                            "rel_l2_vs_exact_adjoint": err,
                            "setting": f"Morton tree, order {ORDER}, theta {theta}, leaf {LEAF}, mixed near pairs"}}
    if bench_case is not None:
        pts, a, bb, gam, rad, w, src, tgt = setup(bench_case)
        run_tree = lambda: engine.tree_sum(src, tgt, model, "raise", "mixed", 128, 3.0, theta, ORDER,  # noqa: E731
                                           LEAF, CLEARANCE, "morton", far_counts=False)
        run_tree_adj = lambda: adjoint.adjoint_tree(pts, a, bb, gam, rad, model, w, precision="mixed",  # noqa: E731
                                                    theta=theta, order=ORDER, leaf_size=LEAF, kind="morton")
        run_tree()
        run_tree_adj()
        torch.cuda.synchronize()
        tree = min(_event_ms(run_tree) for _ in range(5))
        tree_adj = min(_event_ms(run_tree_adj) for _ in range(5))
        out["bench_wake"] = {"workload": f"{src.m} segments x {tgt.n} targets", "tree_forward_ms": tree,
                             "tree_adjoint_ms": tree_adj, "ratio_to_tree_forward": tree_adj / tree}
    return out


def sharded_measure(src, case, rank, world, device, args, dist):
    """One wake split over the ranks by Morton ranges of its targets (segments replicated, no collective on the data
    path): device ms per call as the max over ranks, after warm-up; every rank takes the same collective steps."""
    import torch
    from openfawe_b200 import shard
    model = case["model"]

    def run():
        return shard.sharded_tree_sum(src, case["points"], rank, world, model, "mixed", args.theta, args.order,
                                      args.leaf)

    for _ in range(2):
        run()
    torch.cuda.synchronize()
    times = []
    for _ in range(3):
        dist.barrier()
        times.append(_event_ms(run))
    t = torch.tensor([min(times)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"mode": "targets split by Morton range over ranks, segments replicated", "ms_per_call": float(t.item()),
            "targets_per_rank": len(case["points"]) // world}


def _median_ms(fn, repeat, flush=None):
    """Median CUDA-event time of `fn` over `repeat` calls after one warm-up call (L2 flushed before each if given)."""
    import torch
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(repeat):
        if flush is not None:
            flush.zero_()
        times.append(_event_ms(fn))
    return float(statistics.median(times))


def _golden(name):
    try:
        return np.load(os.path.join(GOLDEN, name))
    except OSError:
        return None


def _digest(case):
    h = hashlib.sha256()
    for key in ("points", "starts", "directions", "lengths", "gamma", "radius"):
        h.update(np.ascontiguousarray(case[key], dtype=np.float64).tobytes())
    return h.hexdigest()


def _dropin_ms(case, tree, cuda, repeat=15):
    """Median wall time of the drop-in cuda_tree_sum from host arrays to host results (the call a caller makes); 15
    calls after two warm-up calls, since a call of a few milliseconds shares the box's host cores with other jobs."""
    from openfawe_b200 import vortex_cuda_tree, wakes
    a = (*wakes.backend_args(case), no_exclusions(len(case["points"])), "raise", tree, cuda)
    for _ in range(2):
        vortex_cuda_tree.cuda_tree_sum(*a)
    times = []
    for _ in range(repeat):
        tick = time.perf_counter()
        vortex_cuda_tree.cuda_tree_sum(*a)
        times.append(1e3 * (time.perf_counter() - tick))
    return float(statistics.median(times))


def c1_measure(device, flush):
    """C1: the 16 x 128 lattice (4,207 segments, Rosenhead-Moore 0.05 m) on 1,024 wing points, FP64 direct sum, against
    the reference's own numba result (tests/golden/direct_lattice.npz) and the oracle's CPU direct sum."""
    from oracle import oracle as O
    from openfawe_b200 import engine, vortex_cuda, wakes
    from openfawe_b200.settings import CudaSettings
    case = wakes.lattice()
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    u, _ = engine.direct(src, tgt, case["model"], "raise", "fp64")
    device_ms = _median_ms(lambda: engine.direct(src, tgt, case["model"], "raise", "fp64"), 20, flush)
    csr = no_exclusions(len(case["points"]))
    e2e = []
    for _ in range(12):
        tick = time.perf_counter()
        vortex_cuda.cuda_sum(*args, csr, "raise", CudaSettings("fp64"))
        e2e.append(1e3 * (time.perf_counter() - tick))
    cpu = []
    for _ in range(5):
        tick = time.perf_counter()
        O.direct_sum(*args, csr, "raise")
        cpu.append(1e3 * (time.perf_counter() - tick))
    out = {"workload": f"lattice 16 x 128, {src.m} segments x {tgt.n} targets, Rosenhead-Moore rc 0.05 m, FP64 "
                       f"direct sum", "device_ms": device_ms, "e2e_ms": float(statistics.median(e2e[2:])),
           "cpu_port_ms": float(statistics.median(cpu)), "cpu_cores": host_cores()}
    g = _golden("direct_lattice.npz")
    if g is not None:
        out["vs_reference_numba"] = errors(u.cpu().numpy(), g["u"])
    return out


def c2_measure(device, flush):
    """C2: the README-shape 468-row wakes (102k segments x 20,570 targets), both variants: the reference's self-test
    sheet and the rotor-ring + wing-sheet mix.  The reference's own tree settings (median tree, order 2, leaf 32, theta
    0.5 and 0.2) in FP64 and mixed, the fifth-order Morton tree at the bench setting, the FP64 direct sum, and the
    reference's CPU tree code (oracle port) on the host cores; errors against the reference's numba direct sum and CPU
    tree (tests/golden/c2_*.npz) where the fixture's inputs match."""
    from openfawe_b200 import engine, wakes
    out = {"readme_468_rows_theta_0.2": README_468}
    cpu_later = []
    for name, make in (("sheet", lambda: wakes.selftest_sheet(468, seed=468)),
                       ("rotor", lambda: wakes.rotor_sheet(468, seed=468, targets=TARGETS))):
        case = make()
        g = _golden(f"c2_{name}.npz")
        if g is not None and str(g["inputs_sha256"]) != _digest(case):
            g = None
        model = case["model"]
        src = engine.Sources(case["starts"], case["directions"], case["lengths"], case["gamma"], case["radius"], device)
        tgt = engine.Targets(case["points"], None, device)
        direct, _ = engine.direct(src, tgt, model, "raise", "fp64")
        direct = direct.cpu().numpy()
        ref_direct = g["direct"] if g is not None else direct
        row = {"segments": src.m, "targets": tgt.n, "core_m": float(case["radius"][0]),
               "fp64_direct_ms": _median_ms(lambda: engine.direct(src, tgt, model, "raise", "fp64"), 3, flush),
               "fp64_direct_vs_reference": errors(direct, ref_direct) if g is not None else None,
               "reference_fixture": g is not None}
        for theta in (0.5, 0.2):
            key = f"t{int(round(theta * 100))}"
            cell = {}
            for precision in ("fp64", "mixed"):
                call = lambda: engine.tree_sum(src, tgt, model, "raise", precision, 128, 3.0, theta, 2, 32,  # noqa
                                               CLEARANCE, "median", far_counts=False)
                u = call()[0].cpu().numpy()
                cell[precision] = {"ms": _median_ms(call, 5, flush), "vs_fp64_direct": errors(u, ref_direct),
                                   "e2e_ms": _dropin_ms(case, CallerTreeSettings(theta, 2, 32, CLEARANCE),
                                                        CallerCudaSettings(precision, 128))}
                if g is not None:
                    cpu = g[key]
                    e, te = np.linalg.norm(u - cpu, axis=1), np.linalg.norm(cpu - ref_direct, axis=1)
                    cell[precision]["vs_reference_cpu_tree"] = {
                        "max_over_max_speed": float(e.max() / np.linalg.norm(cpu, axis=1).max()),
                        "max_over_tree_error_max": float(e.max() / te.max()),
                        "rms_over_tree_error_rms": float(np.sqrt(np.mean(e ** 2)) / np.sqrt(np.mean(te ** 2)))}
            if g is not None:
                cell["reference_numba_tree"] = {"ms_in_fixture_run": 1e3 * float(g[key + "_s"]),
                                                "threads": int(g["threads"]),
                                                "vs_fp64_direct": errors(g[key], ref_direct)}
            row[f"median_order2_theta_{theta}"] = cell
        call = lambda: engine.tree_sum(src, tgt, model, "raise", "mixed", 128, 3.0, THETA, ORDER, LEAF,  # noqa: E731
                                       CLEARANCE, "morton", far_counts=False)
        u = call()[0].cpu().numpy()
        row[f"morton_order{ORDER}_theta_{THETA}_leaf_{LEAF}_mixed"] = {"ms": _median_ms(call, 5, flush),
                                                                         "vs_fp64_direct": errors(u, ref_direct)}
        out[name] = row
        cpu_later.append((row, case, ref_direct))
    # the CPU tree code on every host core last, after every GPU and host-array timing of both wakes
    for row, case, ref_direct in cpu_later:
        for theta in (0.5, 0.2):
            runs = [cpu_tree_call(case, theta) for _ in range(3)]
            row[f"median_order2_theta_{theta}"]["cpu_port"] = {
                "ms": 1e3 * statistics.median(r[0] for r in runs), "cores": host_cores(),
                "vs_fp64_direct": errors(runs[-1][1], ref_direct)}
    return out


def default_path_measure(src, tgt, model, direct_host, flush):
    """The bench wake through the path an unchanged caller of the reference reaches: the median tree at order 2 (leaf
    32, mixed), at the equal-accuracy theta 0.04 and the production theta 0.2."""
    from openfawe_b200 import engine
    out = {}
    for theta in (REF_THETA, 0.2):
        call = lambda: engine.tree_sum(src, tgt, model, "raise", "mixed", 128, 3.0, theta, 2, 32, CLEARANCE,  # noqa
                                       "median", far_counts=False)
        u = call()[0].cpu().numpy()
        out[f"theta_{theta}"] = {"ms": _median_ms(call, 3, flush), "vs_fp64_direct": errors(u, direct_host),
                                 "near_pairs": engine.last_stats(src.device.index)["near_pairs"]}
    return out


def only_run(args, case, src, tgt, device):
    """--only: one call kind, warmup + steps times, for profiler runs; prints its counters."""
    import torch
    from openfawe_b200 import adjoint, engine
    model = case["model"]
    if args.only == "tree":
        fn = lambda: engine.tree_sum(src, tgt, model, "raise", "mixed", 128, 3.0, args.theta, args.order,  # noqa
                                     args.leaf, CLEARANCE, args.kind, far_counts=False)
    elif args.only in ("direct-fp64", "direct-mixed"):
        precision = "fp64" if args.only == "direct-fp64" else "mixed"
        fn = lambda: engine.direct(src, tgt, model, "raise", precision)  # noqa: E731
    else:
        ends = case["nodes"][case["edges"][:, 1]]
        pts, a = torch.as_tensor(case["points"], device=device), torch.as_tensor(case["starts"], device=device)
        bb, gam = torch.as_tensor(ends, device=device), torch.as_tensor(case["gamma"], device=device)
        rad = torch.as_tensor(case["radius"], device=device)
        w = torch.as_tensor(np.random.default_rng(5).standard_normal((len(case["points"]), 3)), device=device)
        if args.only == "adjoint":
            fn = lambda: adjoint.adjoint_direct(pts, a, bb, gam, rad, model, w)  # noqa: E731
        else:
            fn = lambda: adjoint.adjoint_tree(pts, a, bb, gam, rad, model, w, precision="mixed",  # noqa: E731
                                              theta=args.theta, order=args.order, leaf_size=args.leaf,
                                              kind=args.kind)
    for _ in range(args.warmup + args.steps):
        fn()
    torch.cuda.synchronize()
    print(json.dumps({"only": args.only, "stats": engine.last_stats(device), "config": config(case, args)}))


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.reference_gpu_leg:
        return reference_gpu_leg(args)
    import torch
    from openfawe_b200 import engine, vortex_cuda_tree

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local

    case = workload(args.rows)
    model = case["model"]
    segments = tuple(case[k] for k in ("starts", "directions", "lengths", "gamma", "radius"))
    src = engine.Sources(*segments, device)
    tgt = engine.Targets(case["points"], None, device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    # On N GPUs one call is shared by sources (openfawe_b200.shard): this rank holds its Morton range of the segments,
    # builds its own tree over them, evaluates every target, and the partial velocities are summed over the ranks.
    src_step = src
    if world > 1:
        from openfawe_b200 import shard
        mine = shard.source_shards(case["starts"], case["directions"], case["lengths"], world)[rank]
        src_step = engine.Sources(*(a[mine] for a in segments), device)

    def step():
        u, flags, far = engine.tree_sum(src_step, tgt, model, "raise", "mixed", 128, 3.0, args.theta, args.order,
                                        args.leaf, CLEARANCE, args.kind, far_counts=False)
        if world > 1:
            f = flags.to(torch.int32)
            dist.all_reduce(u, op=dist.ReduceOp.SUM)
            dist.all_reduce(f, op=dist.ReduceOp.MAX)
            flags = f.to(torch.int8)
        return u, flags, far

    if args.only:
        if rank == 0:
            only_run(args, case, src, tgt, device)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # plain FP64 GPU direct sum: the accuracy oracle of this run and the time to beat by 10x
    direct, _ = engine.direct(src, tgt, model, "raise", "fp64")
    torch.cuda.synchronize()
    fp64_times = []
    for _ in range(2):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        direct, _ = engine.direct(src, tgt, model, "raise", "fp64")
        e1.record()
        torch.cuda.synchronize()
        fp64_times.append(e0.elapsed_time(e1))
    fp64_ms = min(fp64_times)
    direct_host = direct.cpu().numpy()

    for _ in range(args.warmup):
        out, flags, _ = step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    times, eval_ms, walk_ms, list_ms, far_ms, counters = [], [], [], [], [], []
    with Clocks(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out, flags, _ = step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            s = engine.last_stats(device)
            eval_ms.append(s["evaluate_ms"])
            walk_ms.append(s["walk_ms"])
            list_ms.append(s["list_ms"])
            far_ms.append(s["far_ms"])
            counters.append(s)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clk.summary()
    ms = float(np.mean(times))
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    u = out.cpu().numpy()
    rel_l2 = float(np.linalg.norm(u - direct_host) / np.linalg.norm(direct_host))
    max_err = float(np.max(np.linalg.norm(u - direct_host, axis=1)) / np.max(np.linalg.norm(direct_host, axis=1)))
    s = counters[-1]

    # roofline of the dominant kernel, the near-leaf list kernel (near pairs on the FP32 pipe): algorithmic flops per
    # launch (W_PAIR per near pair) over its CUDA-event time, against the FP32 FMA rate measured on this device in
    # this run; the far-node list kernel (W_FAR per far evaluation) beside it
    kernel_ms = float(np.mean(list_ms))
    far_kernel_ms = float(np.mean(far_ms))
    flops = W_PAIR * s["near_pairs"]
    far_flops = W_FAR[args.order] * s["far_evaluations"]
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    from openfawe_b200 import _lib
    peak_t = ctypes.c_double(0.0)
    _lib.check(_lib.library().bs_fp32_peak(_lib.context(device), ctypes.byref(peak_t)), "bs_fp32_peak")
    peak = float(peak_t.value)
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": LIST_TRAFFIC, "kernel": "tree_list_kernel<mixed, Lamb-Oseen, near leaves>",
                "kernel_ms": kernel_ms, "flops_per_launch": flops,
                "far_kernel": {"kernel": "tree_list_kernel<mixed, Lamb-Oseen, far nodes>", "kernel_ms": far_kernel_ms,
                               "flops_per_launch": far_flops,
                               "achieved": far_flops / (far_kernel_ms * 1e-3) / 1e12 if far_kernel_ms > 0 else None},
                "peak_note": "FP32 FMA throughput measured in this run (bs_fp32_peak); the pair and far-field "
                             "arithmetic runs on the FP32 pipe, neither HBM- nor tensor-core-bound"}

    # End to end, as an unchanged caller of the reference makes the call: host NumPy in, host NumPy out, the
    # reference's own settings objects (here their field-for-field mirrors) at its equal-accuracy setting (order 2,
    # theta 0.04), mapped by install-time options to the benchmarked fifth-order Morton tree.
    e2e, e2e_stages, e2e_effective = [], [], None
    h2d = sum(np.asarray(x).nbytes for x in (case["points"], *segments))
    d2h = len(case["points"]) * (24 + 1 + 8)
    if world == 1:
        import openfawe_b200
        openfawe_b200.install(tree=args.kind, order=args.order, theta={REF_THETA: args.theta}, leaf_size=args.leaf)
        tree = CallerTreeSettings(REF_THETA, REF_ORDER, REF_LEAF, CLEARANCE)
        cuda = CallerCudaSettings("mixed", 128, "gpu64")
        a = (case["points"], *segments, model, no_exclusions(len(case["points"])), "raise", tree, cuda)
        for _ in range(3):  # warm-up: staging ring, pools, host pages
            vortex_cuda_tree.cuda_tree_sum(*a)
        # the median of 10-20 calls: host copies share the box's cores with other jobs, so single calls vary
        for _ in range(max(10, min(2 * args.steps, 20))):
            torch.cuda.synchronize()
            tick = time.perf_counter()
            vortex_cuda_tree.cuda_tree_sum(*a)
            e2e.append(1e3 * (time.perf_counter() - tick))
            last = vortex_cuda_tree.Statistics.last
            e2e_stages.append({k: 1e3 * last[k] for k in ("upload_s", "build_s", "evaluate_s", "download_s")})
        e2e_effective = dict(vortex_cuda_tree.Statistics.last["effective"])
        openfawe_b200.uninstall()
        e2e_call = ("cuda_tree_sum from host arrays with the reference's TreeSettings(theta=0.04, order=2, "
                    "leaf_size=32) and CudaSettings('mixed', 128, 'gpu64'); install-time options map them to the "
                    "effective tree below")
    else:
        # every rank uploads its share of the segments and all targets, evaluates, and reads the summed result back
        from openfawe_b200 import shard
        evaluate = shard.tree_evaluator(model, device, "mixed", args.theta, args.order, args.leaf, kind=args.kind)
        for k in range(2 + max(5, min(args.steps, 10))):
            torch.cuda.synchronize()
            dist.barrier()
            tick = time.perf_counter()
            shard.sharded_sum(evaluate, case["points"], segments, rank, world, "sources")[0].cpu()
            elapsed = torch.tensor([1e3 * (time.perf_counter() - tick)], dtype=torch.float64, device=device)
            dist.all_reduce(elapsed, op=dist.ReduceOp.MAX)
            if k >= 2:
                e2e.append(float(elapsed.item()))
        e2e_effective = dict(tree=args.kind, order=args.order, theta=args.theta, leaf_size=args.leaf)
        e2e_call = (f"openfawe_b200.shard.sharded_sum over {world} ranks from host arrays (each rank uploads its "
                    f"Morton range of the segments and every target), result read back on every rank; wall time, "
                    f"max over ranks")
        h2d = h2d + (world - 1) * case["points"].nbytes
        d2h = world * len(case["points"]) * (24 + 1)

    # launches of this library's kernels inside one step (CUPTI through the torch profiler); the step itself runs on
    # every rank whatever the profiler does, so the ranks' collectives stay matched
    gpu_launches, prof = None, None
    try:
        from torch.profiler import ProfilerActivity, profile
        prof = profile(activities=[ProfilerActivity.CUDA])
        prof.__enter__()
    except Exception:  # noqa: BLE001 - profiler unavailable: leave the count out rather than guess
        prof = None
    step()
    torch.cuda.synchronize()
    if prof is not None:
        try:
            prof.__exit__(None, None, None)
            gpu_launches = sum(1 for e in prof.events() if e.device_type.name == "CUDA" and "bs::" in e.name)
        except Exception:  # noqa: BLE001
            gpu_launches = None

    line = {"metric": METRIC, "value": ms, "unit": "ms/call", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": config(case, args),
            "accuracy": {"rel_l2_vs_fp64_direct": rel_l2, "max_err_over_max_speed": max_err},
            "fp64_direct_ms": fp64_ms, "speedup_vs_fp64_direct": fp64_ms / ms,
            "stages": {"build_ms": s["build_ms"], "moments_ms": s["moments_ms"],
                       "evaluate_ms": float(np.mean(eval_ms)), "walk_ms": float(np.mean(walk_ms)),
                       "list_ms": kernel_ms, "far_ms": far_kernel_ms,
                       "nodes": s["nodes"], "near_pairs": s["near_pairs"], "far_evaluations": s["far_evaluations"],
                       "fp64_pairs": s["fp64_pairs"], "visits": s["visits"]},
            "interactions_per_s": {"executed": (s["near_pairs"] + s["far_evaluations"]) / (ms * 1e-3),
                                   "direct_equivalent": len(case["points"]) * len(case["starts"]) / (ms * 1e-3)},
            "roofline": roofline,
            "e2e": {"value": float(np.median(e2e)), "unit": "ms/call", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "calls_ms": e2e,
                    "stages_ms_of_median_call": (e2e_stages[int(np.argsort(e2e)[len(e2e) // 2])]
                                                 if e2e_stages else None),
                    "call": e2e_call, "effective": e2e_effective},
            "gpu_launches": gpu_launches, "clocks": clocks}
    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(case, direct_host)
        if not args.no_extras:
            line["default_path"] = default_path_measure(src, tgt, model, direct_host, flush)
            line["c1"] = c1_measure(device, flush)
            line["c2"] = c2_measure(device, flush)
            line["batch"] = batch_measure(device, args.theta, args.order)
            line["adjoint"] = adjoint_measure(device, args.theta, case)
            line["adjoint_fwd_ratio"] = line["adjoint"]["tree_adjoint"]["ratio_to_tree_forward"]
            line["reference_gpu"] = reference_gpu_measure()
    if dist:
        line["target_sharded"] = sharded_measure(src, case, rank, world, device, args, dist)
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
