"""GPU tree code (libbs_b200 build + moments + traversal) against the reference's tree code and the oracle.

* Median tree: the arrays of vortex_tree.build_tree element for element; node centres, cores and bounding radii bit
  for bit, moments within 1e-12 node-relative (the reference's GPU-moment bound, tests/test_cuda_moments.py:90-105).
* FP64 evaluation: the accepted nodes equal the CPU's (far counts identical per target) and velocities within
  1e-12 * max|u| of the reference's tree_sum (its GPU self-test allows 1e-10, selftest.py:413).
* Mixed: max and rms error against the CPU tree within 0.1 x the CPU tree's own error against the direct sum (the
  self-test's mixed bound, selftest.py:415-417).
* Morton tree: keys, sort permutation and tree arrays bit-exact against the CPU recomputation (oracle/morton_oracle.c).
"""
import numpy as np
import pytest

from conftest import golden, no_exclusions
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def cuda_settings(precision="fp64", tree="median", block=128, suspect="cpu"):
    from openfawe_b200.settings import CudaSettings
    return CudaSettings(precision, block, suspect, tree=tree)


def tree_settings(theta=0.5, order=2, leaf=32):
    from openfawe_b200.settings import TreeSettings
    return TreeSettings(theta, order, leaf)


def node_relative(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.abs(a).reshape(len(a), -1).max(axis=1)
    diff = np.abs(a - b).reshape(len(a), -1).max(axis=1)
    return np.where(scale > 0, diff / np.where(scale > 0, scale, 1.0), diff)


def grid_segments(nx=30, ny=20, length=0.125):
    """Axis-aligned segments on a grid: exactly representable midpoints with many equal coordinates (ties)."""
    starts = np.array([[i * 0.5, j * 0.25, 0.0] for i in range(nx) for j in range(ny)])
    directions = np.tile([1.0, 0.0, 0.0], (len(starts), 1))
    lengths = np.full(len(starts), length)
    return starts, directions, lengths


def random_segments(seed, count):
    rng = np.random.default_rng(seed)
    starts = rng.random((count, 3)) * [20.0, 5.0, 2.0]
    d = rng.normal(size=(count, 3))
    directions = d / np.linalg.norm(d, axis=1)[:, None]
    lengths = 0.2 + 0.3 * rng.random(count)
    gamma = rng.normal(size=count)
    gamma[::7] = 0.0
    radius = rng.uniform(0.0, 0.08, count)
    return starts, directions, lengths, gamma, radius


def test_median_build_element_for_element(device):
    from openfawe_b200 import engine
    cases = [("random", *random_segments(11, 600)[:3], 8), ("grid", *grid_segments(), 32),
             ("grid-leaf-1", *[a[:200] for a in grid_segments()], 1),
             ("coincident", np.ones((40, 3)), np.tile([0.0, 1.0, 0.0], (40, 1)), np.full(40, 0.5), 4),
             # a cluster of 40 identical segments among 600 others: a node of no extent several levels down (the
             # planned levels are then run again one at a time)
             ("coincident-cluster", *[np.concatenate((x, y)) for x, y in zip(
                 random_segments(12, 600)[:3],
                 (np.full((40, 3), 5.0), np.tile([0.0, 0.0, 1.0], (40, 1)), np.full(40, 0.25)))], 4),
             ("fewer-than-a-leaf", *[a[:5] for a in random_segments(3, 5)[:3]], 32),
             ("longer-than-a-chunk", *random_segments(4, 5000)[:3], 16)]
    for name, starts, directions, lengths, leaf in cases:
        m = len(starts)
        src = engine.Sources(starts, directions, lengths, np.ones(m), np.zeros(m), device)
        tree = engine.build_tree(src, leaf_size=leaf, kind="median")
        got = tree.export()
        _, _, _, mid = O.segment_geometry(starts, directions, lengths, np.ones(m))
        ref = O.build_tree(mid, leaf)
        for key, value in zip(("order", "lo", "hi", "left", "right"), ref[:5]):
            assert np.array_equal(got[key], value), (name, key)
        assert tree.count == ref[5]


def test_moments_against_reference(device):
    from openfawe_b200 import engine
    g = golden("moments.npz")
    for seed in (1, 2, 3):
        p = lambda k: g[f"s{seed}_{k}"]  # noqa: E731
        src = engine.Sources(p("starts"), p("directions"), p("lengths"), p("gamma"), p("radius"), device)
        for tree in (engine.build_tree(src, leaf_size=int(p("leaf")), kind="median"),
                     engine.tree_from_arrays(src, p("order"), p("lo"), p("hi"), p("left"), p("right"))):
            got = tree.export()
            for key in ("order", "lo", "hi", "left", "right", "centre", "core", "bound"):
                assert np.array_equal(got[key], p(key)), (seed, key)
            for key in ("m0", "m1", "m2"):
                assert node_relative(p(key), got[key]).max() <= 1e-12, (seed, key)
            for key, made_of in (("w1", "m1"), ("t2", "m2"), ("w2", "m2")):
                scale = np.abs(p(made_of)).reshape(len(p(made_of)), -1).max(axis=1)
                diff = np.abs(p(key) - got[key]).reshape(len(got[key]), -1).max(axis=1)
                assert np.all(diff <= 1e-12 * scale), (seed, key)
            again = tree.export()
            assert all(np.array_equal(got[k], again[k]) for k in got)


def test_fp64_theta_order_sweep_matches_reference_tree(device):
    from openfawe_b200 import engine
    g = golden("tree_lattice.npz")
    args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(g["points"], None, device)
    tree = engine.build_tree(src, leaf_size=8, kind="median")
    for order in (0, 1, 2):
        for theta in (0.6, 0.4, 0.25, 0.15):
            key = f"o{order}_t{int(theta * 100)}"
            u, flags, far = engine.tree_eval(tree, tgt, 2, "raise", "fp64", theta=theta, order=order)
            u, far = u.cpu().numpy(), far.cpu().numpy()
            _, _, d = O.tree_sum(*args, no_exclusions(len(g["points"])), "raise", theta=theta, order=order,
                                 leaf_size=8, details=True)
            assert np.array_equal(far, d["far"]), key
            assert far.mean() == float(g[key + "_far"])
            scale = np.max(np.linalg.norm(g[key], axis=1))
            assert np.max(np.linalg.norm(u - g[key], axis=1)) <= 1e-12 * scale, key
            assert not flags.cpu().numpy().any()


def test_selftest_sheet_fp64_and_mixed_bounds(device):
    from openfawe_b200.vortex_cuda_tree import cuda_tree_sum, Statistics
    g = golden("tree_selftest.npz")
    args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2,
            (g["ptr"], g["seg"]), "raise")
    norm = lambda v: np.linalg.norm(v, axis=1)  # noqa: E731
    for theta in (0.2, 0.5):
        cpu = g[f"t{int(theta * 100)}"]
        scale = norm(cpu).max()
        tree_error = norm(cpu - g["direct"])
        u, flag = cuda_tree_sum(*args, tree_settings(theta), cuda_settings("fp64"))
        assert flag == bool(g[f"t{int(theta * 100)}_flag"])
        assert norm(u - cpu).max() <= 1e-12 * scale
        assert Statistics.last["nodes"] > 0 and Statistics.last_far_counts.shape == (len(g["points"]),)
        for precision in ("mixed", "fp32"):
            u, flag = cuda_tree_sum(*args, tree_settings(theta), cuda_settings(precision, suspect="gpu64"))
            error = norm(u - cpu)
            assert error.max() <= 0.1 * tree_error.max(), (theta, precision)
            assert np.sqrt(np.mean(error ** 2)) <= 0.1 * np.sqrt(np.mean(tree_error ** 2)), (theta, precision)


def test_morton_keys_order_and_tree_bit_exact(device):
    from openfawe_b200 import engine, wakes
    for case in (wakes.selftest_sheet(30, seed=30), wakes.rotor_sheet(40, seed=7, targets=500)):
        m = len(case["starts"])
        src = engine.Sources(case["starts"], case["directions"], case["lengths"], case["gamma"], case["radius"],
                             device)
        for leaf in (1, 8, 32):
            tree = engine.build_tree(src, leaf_size=leaf, kind="morton")
            keys, order = tree.keys()
            ref = O.morton_tree(case["starts"], case["directions"], case["lengths"], leaf)
            assert np.array_equal(keys, ref["keys"])
            assert np.array_equal(order, ref["order"])
            got = tree.export()
            for key in ("order", "lo", "hi", "left", "right"):
                assert np.array_equal(got[key], ref[key]), (leaf, key)
            assert m == len(got["order"])


def test_morton_tree_evaluation_matches_oracle_on_same_tree(device):
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(60, seed=5, targets=3000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    tree = engine.build_tree(src, leaf_size=16, kind="morton")
    ex = tree.export()
    _, ends, _, _ = O.segment_geometry(*args[1:5])
    quantities = tuple(ex[k] for k in ("centre", "bound", "core", "m0", "m1", "m2", "w1", "t2", "w2"))
    tree_arrays = tuple(ex[k] for k in ("order", "lo", "hi", "left", "right"))
    n = len(case["points"])
    for theta in (0.3, 0.1):
        ref, flags, far, _ = O.tree_velocity(*args[:7], "raise", tree_arrays, quantities, theta, 2, 3.0,
                                             no_exclusions(n)[0], np.zeros(0, dtype=np.int64))
        u, gflags, gfar = engine.tree_eval(tree, tgt, 2, "raise", "fp64", theta=theta)
        assert np.array_equal(gfar.cpu().numpy(), far)
        scale = np.linalg.norm(ref, axis=1).max()
        assert np.max(np.linalg.norm(u.cpu().numpy() - ref, axis=1)) <= 1e-12 * scale


def test_morton_fill_sums_exactly_the_leaves_a_warp_opens(device):
    """Single precisions on a Morton tree: a leaf that one lane of a warp opens is summed exactly for every lane of the
    warp that reached it and accepted it as far (those lanes would otherwise idle beside its pairs).  With 32 targets
    (one warp) that is the reference traversal of each target (checked against the oracle's far counts) with every
    accepted leaf that some target opens moved from its expansion to its exact pair sum.  FP64 keeps the reference's
    decisions."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(40, seed=3, targets=8)
    args = wakes.backend_args(case)
    starts, directions, lengths, gamma, radius, model = args[1:7]
    # one warp of targets on a short line through the wake: neighbours whose near fields overlap in part
    points = starts[len(starts) // 3] + np.outer(np.linspace(-1.5, 1.5, 32), [0.3, 1.0, 0.2]) + [0.0, 0.0, 0.35]
    src = engine.Sources(starts, directions, lengths, gamma, radius, device)
    tgt = engine.Targets(points, None, device)
    tree = engine.build_tree(src, leaf_size=16, kind="morton", order=2)
    ex = tree.export()
    lo, hi, left, right, order = ex["lo"], ex["hi"], ex["left"], ex["right"], ex["order"]
    centre, bound, core = ex["centre"], ex["bound"], ex["core"]
    theta, clearance = 0.6, 3.0

    def walk(x):  # the reference's per-target traversal: accepted nodes and opened leaves
        far, near, stack = [], [], [0]
        while stack:
            j = stack.pop()
            rx, ry, rz = x - centre[j]
            dist = np.sqrt(rx * rx + ry * ry + rz * rz)
            if bound[j] < theta * dist and dist - bound[j] >= clearance * core[j]:
                far.append(j)
            elif left[j] < 0:
                near.append(j)
            else:
                stack += [right[j], left[j]]
        return far, near

    walks = [walk(x) for x in points]
    opened = set(j for _, near in walks for j in near)
    quantities = tuple(ex[k] for k in ("centre", "bound", "core", "m0", "m1", "m2", "w1", "t2", "w2"))
    tree_arrays = tuple(ex[k] for k in ("order", "lo", "hi", "left", "right"))
    ref, _, far_ref, _ = O.tree_velocity(points, *args[1:7], "raise", tree_arrays, quantities, theta, 2, clearance,
                                         no_exclusions(32)[0], np.zeros(0, dtype=np.int64))
    assert [len(f) for f, _ in walks] == list(far_ref)
    expect, moved = ref.copy(), np.zeros(32, dtype=np.int64)
    for t, (far, _) in enumerate(walks):
        for j in far:
            if left[j] < 0 and j in opened:
                ids = order[lo[j]:hi[j]]
                pairs, _ = O.pair_matrix(points[t:t + 1], starts[ids], directions[ids], lengths[ids], radius[ids],
                                         model, False)
                exact = (pairs[0] * gamma[ids][:, None]).sum(axis=0)
                expansion = O.far_velocity(points[t] - centre[j], ex["m0"][j], ex["m1"][j], ex["m2"][j],
                                           ex["w1"][j], ex["t2"][j], ex["w2"][j], 2)
                expect[t] += exact - expansion
                moved[t] += 1
    assert moved.sum() > 0
    scale = np.linalg.norm(expect, axis=1).max()
    for precision in ("mixed", "fp32"):
        u, _, far = engine.tree_eval(tree, tgt, model, "raise", precision, theta=theta)
        assert np.array_equal(far.cpu().numpy(), far_ref - moved), precision
        err = np.linalg.norm(u.cpu().numpy() - expect, axis=1).max()
        assert err <= 1e-5 * scale, (precision, err / scale)
    # the moved leaves change the result well beyond that bound: the check sees them
    assert np.linalg.norm(ref - expect, axis=1).max() > 1e-3 * scale
    u64, _, far64 = engine.tree_eval(tree, tgt, model, "raise", "fp64", theta=theta)
    assert np.array_equal(far64.cpu().numpy(), far_ref)
    assert np.linalg.norm(u64.cpu().numpy() - ref, axis=1).max() <= 1e-12 * np.linalg.norm(ref, axis=1).max()


def test_excluded_segment_never_leaks_through_a_far_node(device):
    from openfawe_b200.vortex_cuda_tree import cuda_tree_sum
    g = golden("tree_lattice.npz")
    starts, directions, lengths, gamma = g["starts"], g["directions"], g["lengths"], g["gamma"]
    radius = np.zeros(len(gamma))
    points = starts[:1] + 0.0
    loud, silent = gamma.copy(), gamma.copy()
    loud[-1], silent[-1] = 1e6, 0.0
    ex = O.exclusion_csr(1, np.array([[0, len(gamma) - 1]]))
    for kind in ("median", "morton"):
        for precision in ("fp64", "mixed"):
            s = cuda_settings(precision, kind)
            t = tree_settings(0.6, 2, 4)
            a, _ = cuda_tree_sum(points, starts, directions, lengths, loud, radius, 0, ex, "zero", t, s)
            b, _ = cuda_tree_sum(points, starts, directions, lengths, silent, radius, 0, ex, "zero", t, s)
            assert np.array_equal(a, b), (kind, precision)
            c, _ = cuda_tree_sum(points, starts, directions, lengths, loud, radius, 0, no_exclusions(1), "zero", t, s)
            assert np.linalg.norm(c - b) > 1e3 * np.linalg.norm(b)


def test_errors_like_the_reference(device):
    from openfawe_b200.vortex_cuda_tree import cuda_tree_sum
    g = golden("tree_lattice.npz")
    args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"])
    csr = no_exclusions(len(g["points"]))
    for model in (3, 4, 5):
        with pytest.raises(ValueError):
            cuda_tree_sum(*args, model, csr, "raise", tree_settings(), cuda_settings())
    fp64_gpu64 = type("S", (), dict(precision="fp64", block=128, suspect="gpu64"))()  # refused by CudaSettings too
    with pytest.raises(ValueError, match="single precisions"):
        cuda_tree_sum(*args, 2, csr, "raise", tree_settings(), fp64_gpu64)
    with pytest.raises(RuntimeError, match="stack overflow"):
        cuda_tree_sum(*args, 2, csr, "raise", tree_settings(0.05, 2, 1), cuda_settings(), stack_size=4)
    u, _ = cuda_tree_sum(*args, 2, csr, "raise", tree_settings(0.05, 2, 1), cuda_settings())
    assert np.all(np.isfinite(u))


def test_singular_target_flags(device):
    from openfawe_b200.vortex_cuda_tree import cuda_tree_sum
    g = golden("tree_lattice.npz")
    starts, directions, lengths = g["starts"], g["directions"], g["lengths"]
    point = (starts[3] + 0.5 * lengths[3] * directions[3])[None]
    args = (point, starts, directions, lengths, g["gamma"], np.zeros(len(lengths)), 0, no_exclusions(1))
    for kind in ("median", "morton"):
        for precision in ("fp64", "mixed"):
            _, flag = cuda_tree_sum(*args, "raise", tree_settings(0.4, 2, 2), cuda_settings(precision, kind))
            assert flag
            _, flag = cuda_tree_sum(*args, "zero", tree_settings(0.4, 2, 2), cuda_settings(precision, kind))
            assert not flag


def test_rotor_sheet_mixed_tree_against_fp64_direct(device):
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(120, seed=11, targets=4000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    direct, _ = engine.direct(src, tgt, 2, "raise", "fp64")
    direct = direct.cpu().numpy()
    for kind in ("median", "morton"):
        tree = engine.build_tree(src, leaf_size=32, kind=kind)
        u, flags, _ = engine.tree_eval(tree, tgt, 2, "raise", "mixed", theta=0.05)
        rel = np.linalg.norm(u.cpu().numpy() - direct) / np.linalg.norm(direct)
        assert rel < 1e-6, (kind, rel)


def test_third_order_expansion_converges_one_order_faster(device):
    """Order 3 (the next term of the reference's Taylor series, an extension beyond its orders 0-2): at each opening
    angle its FP64 error against the direct sum is several times below order 2's, and it shrinks ~theta^4 (order 2:
    ~theta^3).  A tree evaluated at order 3 must have been built for it."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(120, seed=9, targets=4000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    direct, _ = engine.direct(src, tgt, 2, "raise", "fp64")
    direct = direct.cpu().numpy()
    err = {}
    for order in (2, 3):
        tree = engine.build_tree(src, leaf_size=16, kind="morton", order=order)
        for theta in (0.1, 0.2):
            u, flags, _ = engine.tree_eval(tree, tgt, 2, "raise", "fp64", theta=theta, order=order)
            assert not flags.cpu().numpy().any()
            err[order, theta] = np.linalg.norm(u.cpu().numpy() - direct) / np.linalg.norm(direct)
    for theta in (0.1, 0.2):
        assert err[3, theta] < 0.35 * err[2, theta], err
    assert err[3, 0.2] / err[3, 0.1] > 8.0 and err[2, 0.2] / err[2, 0.1] > 4.0, err
    with pytest.raises(ValueError):
        engine.tree_eval(engine.build_tree(src, leaf_size=16, kind="morton", order=2), tgt, 2, "raise", "fp64",
                         theta=0.1, order=3)


def test_fourth_order_expansion_converges_one_order_faster_again(device):
    """Order 4 (the fourth moments of the segments' line integrals, an extension beyond the reference's orders 0-2):
    below order 3 at each opening angle, shrinking ~theta^5, on Morton and median trees (both take their fourth-order
    moments bottom-up) and in mixed precision; an order-4 tree evaluated at order 3 matches an order-3 tree."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(120, seed=9, targets=4000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    direct, _ = engine.direct(src, tgt, 2, "raise", "fp64")
    direct = direct.cpu().numpy()
    rel = lambda u: np.linalg.norm(u.cpu().numpy() - direct) / np.linalg.norm(direct)
    for kind in ("morton", "median"):
        err = {}
        trees = {order: engine.build_tree(src, leaf_size=16, kind=kind, order=order) for order in (3, 4)}
        for order in (3, 4):
            for theta in (0.1, 0.2):
                u, flags, _ = engine.tree_eval(trees[order], tgt, 2, "raise", "fp64", theta=theta, order=order)
                assert not flags.cpu().numpy().any()
                err[order, theta] = rel(u)
        for theta in (0.1, 0.2):
            assert err[4, theta] < 0.5 * err[3, theta], (kind, err)
        assert err[4, 0.2] / err[4, 0.1] > 12.0, (kind, err)
        u3, _, _ = engine.tree_eval(trees[4], tgt, 2, "raise", "fp64", theta=0.2, order=3)
        assert abs(rel(u3) - err[3, 0.2]) <= 1e-3 * err[3, 0.2], (kind, rel(u3), err[3, 0.2])
        um, _, _ = engine.tree_eval(trees[4], tgt, 2, "raise", "mixed", theta=0.2, order=4)
        assert rel(um) < 1.5 * err[4, 0.2] + 2e-7, (kind, rel(um), err)
    with pytest.raises(ValueError):
        engine.tree_eval(engine.build_tree(src, leaf_size=16, kind="morton", order=3), tgt, 2, "raise", "fp64",
                         theta=0.1, order=4)


def test_fifth_order_expansion_converges_one_order_faster_again(device):
    """Order 5 (the fifth moments, an extension beyond the reference's orders 0-2; its means come from the three-point
    Gauss-Legendre rule, exact for degree 5).  One cluster of segments seen from b/r = 0.3, 0.2, 1/4, 1/8 (the root
    accepted): from order 1 on, each order's relative error falls by about b/r (at most 1.5 b/r), the mixed far field
    agrees with FP64 to 1e-6 of the field, and a tree of 3-segment leaves (the root's moments translated up from ten leaves) gives the same field as a single leaf.  On the
    rotor sheet without cores (a far node's expansion is that of singular segments: with cores, the far field differs
    from the regularised pairs by an order-independent amount that would hide the comparison): below order 4 at each
    opening angle, shrinking ~theta^6, Morton and median; a fifth-order tree evaluated at order 4 matches a
    fourth-order tree."""
    from openfawe_b200 import engine, wakes
    rng = np.random.default_rng(3)
    m = 30
    starts = rng.normal(scale=0.3, size=(m, 3))
    d = rng.normal(size=(m, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    lengths, gamma, radius = 0.05 + 0.2 * rng.random(m), rng.normal(size=m), np.zeros(m)
    ends = starts + d * lengths[:, None]
    c = 0.5 * (np.minimum(starts, ends).min(0) + np.maximum(starts, ends).max(0))
    b = np.sqrt(np.max(np.sum((np.vstack([starts, ends]) - c) ** 2, axis=1)))
    direction = np.array([0.3, -0.7, 0.5]) / np.linalg.norm([0.3, -0.7, 0.5])
    ratios = np.array([0.3, 0.2, 0.25, 0.125])
    pts = c + (b / ratios)[:, None] * direction
    exact = np.array([(O.pair_matrix(p[None], starts, d, lengths, radius, 0, False)[0][0] * gamma[:, None]).sum(0)
                      for p in pts])
    src = engine.Sources(starts, d, lengths, gamma, radius, device)
    tgt = engine.Targets(pts, None, device)
    for kind in ("morton", "median"):
        fields = {}
        for leaf in (64, 3):
            tree = engine.build_tree(src, leaf_size=leaf, kind=kind, order=5)
            err = []
            for order in range(6):
                u, _, far = engine.tree_eval(tree, tgt, 0, "zero", "fp64", theta=0.5, order=order, clearance=0.0)
                assert np.array_equal(far.cpu().numpy(), np.ones(4)), (kind, leaf)
                fields[leaf, order] = u.cpu().numpy()
                err.append(np.linalg.norm(fields[leaf, order] - exact, axis=1) / np.linalg.norm(exact, axis=1))
                # the single-precision far field (on the unit vector) agrees with FP64 to FP32 rounding
                um, _, _ = engine.tree_eval(tree, tgt, 0, "zero", "mixed", theta=0.5, order=order, clearance=0.0)
                gap = np.linalg.norm(um.cpu().numpy() - fields[leaf, order], axis=1) / np.linalg.norm(exact, axis=1)
                assert np.all(gap < 1e-6), (kind, leaf, order, gap)
            assert np.all(err[1] < err[0]), (kind, leaf, err)
            for order in range(1, 5):
                assert np.all(err[order + 1] < 1.5 * ratios * err[order]), (kind, leaf, order, err)
        for order in range(6):
            np.testing.assert_allclose(fields[3, order], fields[64, order], rtol=1e-10, atol=0)
    case = wakes.rotor_sheet(120, seed=9, targets=4000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:5], np.zeros(len(args[4])), device)
    tgt = engine.Targets(case["points"], None, device)
    direct, _ = engine.direct(src, tgt, 0, "zero", "fp64")
    direct = direct.cpu().numpy()
    rel = lambda u: np.linalg.norm(u.cpu().numpy() - direct) / np.linalg.norm(direct)
    for kind in ("morton", "median"):
        err = {}
        trees = {order: engine.build_tree(src, leaf_size=16, kind=kind, order=order) for order in (4, 5)}
        for order in (4, 5):
            for theta in (0.1, 0.2):
                u, _, _ = engine.tree_eval(trees[order], tgt, 0, "zero", "fp64", theta=theta, order=order)
                err[order, theta] = rel(u)
        for theta in (0.1, 0.2):
            assert err[5, theta] < 0.5 * err[4, theta], (kind, err)
        assert err[5, 0.2] / err[5, 0.1] > 20.0, (kind, err)
        u4, _, _ = engine.tree_eval(trees[5], tgt, 0, "zero", "fp64", theta=0.2, order=4)
        assert abs(rel(u4) - err[4, 0.2]) <= 1e-3 * err[4, 0.2], (kind, rel(u4), err[4, 0.2])
    with pytest.raises(ValueError):
        engine.tree_eval(engine.build_tree(src, leaf_size=16, kind="morton", order=4), tgt, 2, "raise", "fp64",
                         theta=0.1, order=5)


def test_morton_bottom_up_moments_against_direct_node_sums(device):
    """Morton trees and forests take their node moments bottom-up (leaves summed, parents translated from their
    children): box, centre, core and bounding radius equal the direct per-node computation bit for bit, the moments
    agree to rounding (1e-12 of the node's largest child-moment magnitude)."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(80, seed=11, targets=10)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    starts = args[1]
    lv, ends, alpha, _ = O.segment_geometry(*args[1:5])
    for leaf in (1, 8, 32):
        tree = engine.build_tree(src, leaf_size=leaf, kind="morton")
        ex = tree.export()
        ref = O.node_moments(ex["order"], ex["lo"], ex["hi"], starts, ends, alpha, lv, args[5], args[4])
        for key, value in zip(("centre", "bound", "core"), ref[:3]):
            assert np.array_equal(ex[key], value), (leaf, key)
        # translation rounds like a sum over the node's segments: scale by the segments' own moment magnitudes
        seg_scale = np.abs(alpha).max() * (1.0 + np.abs(ex["bound"]).max()) ** 2
        for key, value in zip(("m0", "m1", "m2"), ref[3:]):
            assert np.abs(ex[key] - value).max() <= 1e-12 * seg_scale * len(starts), (leaf, key)
            assert node_relative(value, ex[key]).max() <= 1e-9, (leaf, key)


def test_list_overflow_is_evaluated_by_the_walk(device):
    """A warp whose interaction list outgrows its chunk table (4,096 entries) or the shared pool evaluates the rest in
    the walk itself: results stay as close to the direct sum as the truncation allows."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(60, seed=13, targets=2000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    direct, _ = engine.direct(src, tgt, 2, "raise", "fp64")
    direct = direct.cpu().numpy()
    tree = engine.build_tree(src, leaf_size=1, kind="morton")
    for precision, bound in (("fp64", 1e-6), ("mixed", 1e-6)):  # truncation at theta 0.02 is ~5e-8
        u, flags, far = engine.tree_eval(tree, tgt, 2, "raise", precision, theta=0.02)
        # thousands of entries per warp of targets: far beyond one warp's list.  In FP64 one target's far count shows
        # it; in single precision a one-segment leaf that the warp opens for one lane is summed exactly by the lanes
        # that accepted it, so count the near entries (one a leaf, 32 lane slots each) per warp instead
        near_entries = engine.last_stats(device)["pair_slots"] / 32 / ((len(case["points"]) + 31) // 32)
        assert int(far.cpu().numpy().max()) > 4096 or near_entries > 4096, (precision, near_entries)
        rel = np.linalg.norm(u.cpu().numpy() - direct) / np.linalg.norm(direct)
        assert rel < bound and not flags.cpu().numpy().any(), (precision, rel)


def test_list_overflow_while_far_records_are_pending(device):
    """A tree sum computes the far records on a side stream beside the walk; a walk whose list overflowed onto a far
    node before they were complete is evaluated again once they are: device and host tree sums equal a separate build
    and evaluation bit for bit, with thousands of far entries per warp (far beyond one list)."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(60, seed=13, targets=2000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    for kind, order in (("morton", 2), ("median", 4)):
        tree = engine.build_tree(src, leaf_size=1, kind=kind, order=order)
        ref, ref_flags, far = engine.tree_eval(tree, tgt, 2, "raise", "mixed", theta=0.02, order=order)
        # far beyond one warp's list: shown by a target's far count or (Morton trees sum the leaves a warp opens for
        # every lane that reached them) by the near entries a warp, one a one-segment leaf
        near_entries = engine.last_stats(device)["pair_slots"] / 32 / ((len(case["points"]) + 31) // 32)
        assert int(far.cpu().numpy().max()) > 4096 or near_entries > 4096, (kind, near_entries)
        u, flags, _ = engine.tree_sum(src, tgt, 2, "raise", "mixed", 128, 3.0, 0.02, order, 1, 3.0, kind)
        assert np.array_equal(u.cpu().numpy(), ref.cpu().numpy()), (kind, order)
        assert np.array_equal(flags.cpu().numpy(), ref_flags.cpu().numpy())
        uh, _, _ = engine.tree_sum_host(case["points"], *args[1:6], None, 2, "raise", "mixed", 128, 3.0, 0.02, order,
                                        1, 3.0, kind, device=device)
        assert np.array_equal(uh, ref.cpu().numpy()), (kind, order)


def test_upload_moves_host_bytes_exactly(device):
    """bs_upload (pinned staging ring, threaded host copies) delivers every byte, for sizes around its chunk size."""
    import torch
    from openfawe_b200 import engine
    rng = np.random.default_rng(17)
    for count in (1 << 17, (4 << 20) // 8 + 3, (12 << 20) // 8 - 5):
        host = rng.normal(size=count)
        dev = engine.f64(host, torch.device("cuda", device))
        assert np.array_equal(dev.cpu().numpy(), host)


def test_upload_many_moves_every_array_exactly(device):
    """bs_upload_many (one pass of the staging ring over several arrays, non-temporal staging copies) delivers every
    byte of each array, for sizes that end inside, at and across chunk boundaries, with small arrays in between."""
    import torch
    from openfawe_b200 import engine
    rng = np.random.default_rng(19)
    sizes = ((4 << 20) // 8, 3, (1 << 20) // 8 + 1, (9 << 20) // 8 - 7, 1 << 17, (4 << 20) // 8 + 5)
    hosts = [rng.normal(size=c) for c in sizes]
    hosts.append(np.asfortranarray(rng.normal(size=(70000, 3))))  # not C-contiguous: copied first
    for _ in range(2):
        devs = engine.f64_many(hosts, torch.device("cuda", device))
        for h, d in zip(hosts, devs):
            assert np.array_equal(d.cpu().numpy(), np.ascontiguousarray(h))


def test_download_many_moves_every_array_exactly(device):
    """bs_download_many (device -> host through the pinned ring, the next chunk in flight while the previous one is
    copied out) returns every byte, for arrays that end inside, at and across chunk boundaries and of several types."""
    import torch
    from openfawe_b200 import engine
    rng = np.random.default_rng(23)
    dev = torch.device("cuda", device)
    arrays = [rng.normal(size=(4 << 20) // 8), rng.normal(size=3), rng.integers(-9, 9, size=(9 << 20) + 5).astype(np.int8),
              rng.integers(0, 1 << 40, size=(1 << 17) + 1), rng.normal(size=((17 << 20) // 24, 3))]
    tensors = [torch.as_tensor(a, device=dev) for a in arrays]
    for _ in range(2):
        got = engine.to_host_many(tensors + [None], [a.shape for a in arrays] + [(1,)],
                                  [a.dtype for a in arrays] + [np.float64])
        assert got[-1] is None
        for a, g in zip(arrays, got):
            assert g.dtype == a.dtype and np.array_equal(g, a)


def test_tree_sum_from_host_arrays_equals_device_call(device):
    """bs_tree_sum_host (host arrays in and out; circulations and cores uploaded while the Morton keys are sorted)
    returns exactly what bs_tree_sum returns on the same inputs, for Morton and median trees, with and without
    exclusions, twice in a row; no segments gives zeros."""
    from openfawe_b200 import engine, wakes
    g = golden("tree_selftest.npz")
    sheet = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"])
    rotor = wakes.rotor_sheet(60, seed=5, targets=3000)
    cases = [(sheet, (g["ptr"], g["seg"])), (wakes.backend_args(rotor)[:6], None)]
    for (points, starts, directions, lengths, gamma, radius), csr in cases:
        src = engine.Sources(starts, directions, lengths, gamma, radius, device)
        tgt = engine.Targets(points, csr, device)
        for kind, order, leaf in (("morton", 4, 64), ("median", 2, 16)):
            for _ in range(2):
                ref = engine.tree_sum(src, tgt, 2, "zero", "mixed", 128, 3.0, 0.3, order, leaf, 3.0, kind)
                got = engine.tree_sum_host(points, starts, directions, lengths, gamma, radius, csr, 2, "zero",
                                           "mixed", 128, 3.0, 0.3, order, leaf, 3.0, kind, 0, device)
                for r, h in zip(ref, got):
                    assert np.array_equal(r.cpu().numpy(), h), (kind, order)
    u, flags, far = engine.tree_sum_host(np.ones((5, 3)), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0),
                                         np.zeros(0), np.zeros(0), None, 2, device=device, kind="morton")
    assert np.all(u == 0) and not flags.any() and not far.any()


def test_mixed_tree_far_field_at_any_length_scale(device):
    """The single-precision far field is formed on the unit vector with one power of 1/r per order, so the same wake
    at 1e-4, 1 and 1e4 times its size (cores scaled with it) gives the same relative error against the FP64 direct sum
    at orders 2, 4 and 5 (r^-13 itself would leave FP32's range at both ends)."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(40, seed=21, targets=1500)
    args = wakes.backend_args(case)
    errs = {}
    for scale in (1.0, 1e-4, 1e4):
        pts, st, dr, ln, gm, rc = args[0] * scale, args[1] * scale, args[2], args[3] * scale, args[4], args[5] * scale
        src = engine.Sources(st, dr, ln, gm, rc, device)
        tgt = engine.Targets(pts, None, device)
        direct, _ = engine.direct(src, tgt, 2, "raise", "fp64")
        direct = direct.cpu().numpy()
        for order in (2, 4, 5):
            u, flags, _ = engine.tree_sum(src, tgt, 2, "raise", "mixed", 128, 3.0, 0.3, order, 32, 3.0, "morton")
            u = u.cpu().numpy()
            assert np.all(np.isfinite(u)) and not flags.cpu().numpy().any(), (scale, order)
            errs[scale, order] = np.linalg.norm(u - direct) / np.linalg.norm(direct)
    for order in (2, 4, 5):
        for scale in (1e-4, 1e4):
            assert errs[scale, order] <= 1.1 * errs[1.0, order] + 1e-7, errs


@pytest.mark.parametrize("model", [0, 1, 2])
def test_single_precision_near_field_every_packed_model(device, model):
    """The packed near-field forms (the clear-leaf pair for targets 1.5 bounding radii out, pair32x2 nearer, the
    scalar pair at the leaves' odd ends) for the no-core, Rankine and Lamb-Oseen models: a fifth-order Morton tree at
    theta 0.1 and leaf 128 in mixed and FP32 against the FP64 direct sum.  The targets sit 0.011 m above the sheet's
    nodes, 0.05 segment lengths from the nodes' segments: the cores' FP64 rule (3 core radii) covers them for models 1
    and 2, the no-core rule (within L/4 of the segment) for model 0, which without it erred by 2.3e-6."""
    from openfawe_b200 import engine, wakes
    case = wakes.rotor_sheet(40, seed=21 + model, targets=2000)
    args = wakes.backend_args(case)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(case["points"], None, device)
    ref, rflags = engine.direct(src, tgt, model, "zero", "fp64")
    ref = ref.cpu().numpy()
    assert not rflags.cpu().numpy().any()
    tree = engine.build_tree(src, theta=0.1, order=5, leaf_size=128, kind="morton")
    for precision, bound in (("mixed", 2e-8 if model == 0 else 3e-7), ("fp32", 5e-7)):
        u, flags, _ = engine.tree_eval(tree, tgt, model, "zero", precision, theta=0.1, order=5)
        rel = np.linalg.norm(u.cpu().numpy() - ref) / np.linalg.norm(ref)
        assert rel <= bound and not flags.cpu().numpy().any(), (model, precision, rel)
        assert engine.last_stats(device)["fp64_pairs"] > 0
