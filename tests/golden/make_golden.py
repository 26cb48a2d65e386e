"""Generate the golden fixtures of tests/golden/ by running the reference's own code.

Run in a container that holds the reference project (read-only); give its location with --reference or the
OPENFAWE_REFERENCE environment variable:

    python tests/golden/make_golden.py --reference <path of the reference project> [--only NAME]

It imports the reference's numba backends (src/openfawe/aero/vortex_numba.py, vortex_tree.py) with the numba cache
redirected outside the reference tree, evaluates them on small seeded cases and writes compressed ``.npz`` files beside
this script.  The GPU box does not have the reference; the tests only read these files.
"""
import argparse
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path)} bytes")


def random_network(seed, nodes=60, segments=90, points=70):
    """Random directed network with near-axis, collinear-exterior and off-line targets (the kind of case that
    tests/test_vortex_numba.py:38-54 of the reference uses)."""
    rng = np.random.default_rng(seed)
    xyz = rng.normal(size=(nodes, 3))
    edges = rng.integers(0, nodes, size=(segments, 2))
    edges = edges[edges[:, 0] != edges[:, 1]]
    gamma = rng.normal(size=len(edges))
    gamma[::7] = 0.0
    radius = rng.uniform(0.01, 0.6, size=len(edges))
    targets = rng.normal(size=(points, 3))
    a, b = xyz[edges[:5, 0]], xyz[edges[:5, 1]]
    normal = np.cross(b - a, [0.3, -0.2, 0.9])
    normal /= np.linalg.norm(normal, axis=1)[:, None]
    near = [a + 0.4 * (b - a) + 1e-9 * normal, a + 0.4 * (b - a) + 1e-13 * normal, a + 1.7 * (b - a),
            a - 0.5 * (b - a), a + 0.5 * (b - a) + 0.05 * normal]
    return xyz, edges, gamma, radius, np.vstack([targets, *near])


def segment_arrays(nodes, edges):
    """starts, directions, lengths exactly as segments_velocity forms them (vortex.py:460-465)."""
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
    return starts, delta / lengths[:, None], lengths


def input_digest(case):
    """SHA-256 over the bytes of a case's backend inputs (points, starts, directions, lengths, gamma, radius)."""
    import hashlib
    h = hashlib.sha256()
    for key in ("points", "starts", "directions", "lengths", "gamma", "radius"):
        h.update(np.ascontiguousarray(case[key], dtype=np.float64).tobytes())
    return h.hexdigest()


def ring_lattice(seed=11, rows=24, span=17):
    """A wavy ring lattice with shed circulation differences (the case family of tests/test_vortex_tree.py:25-40)."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, 12.0, rows)[:, None] * np.ones((1, span))
    y = np.ones((rows, 1)) * np.linspace(-4.0, 4.0, span)[None, :]
    z = 0.3 * np.sin(0.7 * x) * np.cos(0.5 * y) + 0.05 * rng.normal(size=x.shape)
    nodes = np.column_stack((x.ravel(), y.ravel(), z.ravel()))
    edges, gamma = [], []
    strength = np.cos(np.linspace(-1.3, 1.3, span - 1))[None, :] * np.exp(-0.05 * np.arange(rows - 1))[:, None]
    for i in range(rows - 1):
        for j in range(span - 1):
            a, b, c, d = i * span + j, i * span + j + 1, (i + 1) * span + j + 1, (i + 1) * span + j
            for p, q in ((a, b), (b, c), (c, d), (d, a)):
                edges.append((p, q))
                gamma.append(strength[i, j])
    return nodes, np.asarray(edges, dtype=np.int64), np.asarray(gamma)


def network_cases(seed):
    """Wake networks whose free nodes (index >= first) coincide bit for bit with bound nodes and with each other, plus
    -0.0 / 0.0 twins, NaN and infinite coordinates (the cases network_numba.py:13-22 of the reference describes)."""
    rng = np.random.default_rng(seed)
    bound = np.round(rng.normal(size=(40, 3)), 2)
    bound[3] = [0.0, 1.0, 2.0]
    free = np.round(rng.normal(size=(120, 3)), 2)
    pick = rng.integers(0, 40, 50)
    free[:50] = bound[pick]                      # shed nodes sitting on bound nodes
    free[50:80] = free[rng.integers(0, 50, 30)]  # repeated free nodes
    free[80] = [-0.0, 1.0, 2.0]                  # differs from bound[3] only in the sign of zero
    free[81] = [0.0, 1.0, 2.0]
    free[82] = [np.nan, 0.5, 0.5]
    free[83] = [np.nan, 0.5, 0.5]
    free[84] = [np.inf, -1.0, 0.0]
    free[85] = [np.inf, -1.0, 0.0]
    nodes = np.vstack([bound, free])
    edges = rng.integers(0, len(nodes), size=(300, 2))
    edges[:6] = [[3, 120], [122, 123], [124, 125], [40 + 84, 40 + 85], [0, 40], [40 + 81, 3]]
    return nodes, edges.astype(np.int64), len(bound)


def exclusion_cases(seed):
    rng = np.random.default_rng(seed)
    points = rng.integers(0, 50, 400)
    segments = rng.integers(0, 30, 400)
    out = {"a": (60, np.column_stack((points, segments)))}
    # repeats, negative and very large segment ids, unused trailing points
    b = np.column_stack((rng.integers(0, 7, 90), rng.choice([-5, -1, 0, 3, 2**40, 2**62, 17], 90)))
    out["b"] = (12, b)
    out["c"] = (5, np.zeros((0, 2), dtype=np.int64))
    out["d"] = (3, np.array([[2, 9], [2, 9], [0, 4], [2, 1]]))
    return out


def main():
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("OPENFAWE_REFERENCE"),
                        help="the reference project's root (default: $OPENFAWE_REFERENCE)")
    parser.add_argument("--only", default=None, help="write only this fixture (e.g. network.npz)")
    args = parser.parse_args()
    if not args.reference:
        parser.error("give the reference project's root with --reference or OPENFAWE_REFERENCE")
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "numba_reference_cache"))
    sys.path.insert(0, os.path.join(args.reference, "src"))
    sys.path.insert(0, REPO)
    from openfawe.aero import vortex_numba as vn, vortex_tree as vt
    from openfawe_b200 import wakes

    if args.only == "convection.npz" or args.only is None:
        # one step of the reference's geometry convection stages (wake._network_convection, wake.py:404-491) on a
        # rotor-sheet network whose first row is the bound row; the integrators combine the stages as
        # wake.convect_geometry does (wake.py:590-606)
        import types
        from openfawe.aero import wake as W
        from openfawe.aero.vortex import CoreModel
        case = wakes.rotor_sheet(10, seed=10, targets=1)
        nodes, edges = case["nodes"], case["edges"]
        first = 174
        gamma = np.random.default_rng(10).uniform(0.0, 8.0, len(edges))
        radii = np.full(len(edges), 0.05)
        config = types.SimpleNamespace(free_wake=True, velocity_backend="numba", core_model=CoreModel.LAMB_OSEEN)
        inflow = np.array([10.0, 0.0, 0.5])
        dt = 0.02

        def rhs(points, t):
            return W._network_convection(np.concatenate((nodes[:first], points)), edges, gamma, first, radii, config,
                                         inflow, t)
        out = dict(nodes=nodes, edges=edges, gamma=gamma, radii=radii, first=np.array(first), inflow=inflow,
                   dt=np.array(dt))
        points = nodes[first:].copy()
        k1 = rhs(points, 0.0)
        out["k1"] = k1
        out["euler"] = points + dt * k1
        k2 = rhs(points + dt * k1, dt)
        out["heun"] = points + dt * (k1 + k2) / 2
        k2 = rhs(points + dt * k1 / 2, dt / 2)
        k3 = rhs(points + dt * k2 / 2, dt / 2)
        k4 = rhs(points + dt * k3, dt)
        out["rk4"] = points + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6
        save("convection.npz", **out)
        if args.only:
            return

    if args.only == "convection_rings.npz" or args.only is None:
        # one stage of wake._network_convection (wake.py:404-491) on a network with rotor rings after its wing rows:
        # the rotor-sheet network reordered so that every ring node follows every wing node, the first wing row
        # bound; five settings: rows and rings; the leading ring nodes free, the ring targets with their own cores;
        # the far-wake row limit with frozen rows at the ambient flow; the same with the frozen rows drifting with
        # the rings' induction; all of these at once
        import types
        from openfawe.aero import wake as W
        from openfawe.aero.vortex import CoreModel
        case = wakes.rotor_sheet(6, seed=12, targets=1)
        per_row, wing = 46 + 8 * 16, 46
        index = np.arange(len(case["nodes"]))
        is_wing = (index % per_row) < wing
        order = np.concatenate((index[is_wing], index[~is_wing]))
        position = np.empty_like(order)
        position[order] = np.arange(len(order))
        nodes = case["nodes"][order]
        edges = position[case["edges"]]
        first, ring_first = wing, int(is_wing.sum())
        rng = np.random.default_rng(12)
        gamma = rng.uniform(0.0, 8.0, len(edges))
        radii = np.full(len(edges), 0.05)
        ring_radii = np.full(len(edges), 0.08)
        inflow = np.array([10.0, 0.0, 0.5])
        out = dict(nodes=nodes, edges=edges, gamma=gamma, radii=radii, ring_radii=ring_radii, first=np.array(first),
                   ring_first=np.array(ring_first), inflow=inflow)
        settings = {"rings": dict(), "ring_free": dict(ring_free=200, ring_radii=ring_radii),
                    "row_limit": dict(rows=3, drift="ambient"), "row_limit_rings": dict(rows=3, drift="ambient_rings"),
                    "all": dict(ring_free=200, ring_radii=ring_radii, rows=3, drift="ambient_rings")}
        for name, opt in settings.items():
            config = types.SimpleNamespace(free_wake=True, velocity_backend="numba", core_model=CoreModel.LAMB_OSEEN)
            if "rows" in opt:
                config.free_convection_rows = opt["rows"]
                config.frozen_rows_drift = opt["drift"]
            out[name] = W._network_convection(nodes, edges, gamma, first, radii, config, inflow, 0.0,
                                              ring_first=ring_first, ring_free=opt.get("ring_free"),
                                              ring_radii=opt.get("ring_radii"))
        save("convection_rings.npz", **out)
        if args.only:
            return

    if args.only == "frozen_state.npz" or args.only is None:
        # a frozen state in the benchmark's format and the reference's own segments_velocity on it (the numba direct
        # sum the benchmark takes as its reference, local_benchmark.py:56-66)
        from openfawe.aero.vortex import segments_velocity
        from openfawe.aero.network_numba import incident_pairs
        from openfawe_b200 import wakestate
        case = wakes.rotor_sheet(24, seed=24, targets=1)
        nodes, edges = case["nodes"], case["edges"]
        first = 174
        gamma = np.random.default_rng(24).uniform(0.0, 8.0, len(edges))
        radii = np.random.default_rng(25).uniform(0.03, 0.08, len(edges))
        exclusions = incident_pairs(nodes, edges, first)
        path = os.path.join(HERE, "frozen_state_input.npz")
        wakestate.save_state(path, nodes, edges, gamma, radii, first, 10.0, 2, exclusions)
        u = segments_velocity(nodes[first:], nodes, edges, gamma, model=2, core_radius=radii, exclusions=exclusions,
                              backend="numba")
        save("frozen_state.npz", u=u)
        if args.only:
            return

    if args.only == "operators.npz" or args.only is None:
        out = {}
        wing = wakes.ring_wing(panels=16, rows=3)
        rng = np.random.default_rng(8)
        # control points, points on the bound line and on a trailing segment (flagged pairs), off-wing points
        a, b = wing["nodes"][wing["edges"][:3, 0]], wing["nodes"][wing["edges"][:3, 1]]
        points = np.vstack([wing["points"], a + 0.5 * (b - a), a, rng.normal(scale=5.0, size=(8, 3))])
        for model in (0, 2, 5):
            for raise_singular in (True, False):
                radius = wing["radius"] if model else np.zeros(len(wing["radius"]))
                pairs = np.zeros((len(points), len(wing["starts"]), 3))
                flags = np.zeros(len(points), dtype=np.int8)
                vn.pair_matrix(points, wing["starts"], wing["directions"], wing["lengths"], radius, model,
                               raise_singular, pairs, flags)
                cols = np.zeros((len(points), len(wing["column_ptr"]) - 1, 3))
                vn.assemble_columns(pairs, wing["column_ptr"], wing["column_segment"], wing["column_sign"], cols)
                key = f"m{model}_{'raise' if raise_singular else 'zero'}"
                out[key + "_pairs"], out[key + "_flags"], out[key + "_columns"] = pairs, flags, cols
        out["points"] = points
        save("operators.npz", **out)
        if args.only:
            return

    for name, make in (("c2_sheet.npz", lambda: wakes.selftest_sheet(468, seed=468)),
                       ("c2_rotor.npz", lambda: wakes.rotor_sheet(468, seed=468, targets=20570))):
        if args.only not in (name, None):
            continue
        # Full-size C2 wakes (102k segments x 20,570 targets): the reference's numba direct sum and its CPU tree code
        # at the reference default (theta 0.5) and the production setting (theta 0.2), order 2, leaf 32, clearance 3
        # (vortex.py:30-55; apps/studio/openfawe_studio/selftest.py:35).  The inputs come from this repository's
        # generators; their SHA-256 is stored so that a test can check it regenerated the same arrays.
        import time
        import numba
        case = make()
        args_ = wakes.backend_args(case)
        csr = vn.exclusion_csr(len(case["points"]), np.zeros((0, 2), dtype=np.int64))
        out = dict(inputs_sha256=np.array(input_digest(case)), threads=np.array(numba.get_num_threads()))
        vn.direct_sum(args_[0][:64], *args_[1:], (csr[0][:65], csr[1]), "raise")   # compile
        tick = time.perf_counter()
        out["direct"], flagged = vn.direct_sum(*args_, csr, "raise")
        out["direct_s"], out["direct_flag"] = np.array(time.perf_counter() - tick), np.array(flagged)
        for theta in (0.5, 0.2):
            settings = type("S", (), dict(theta=theta, order=2, leaf_size=32, core_clearance=3.0))()
            vt.tree_sum(*args_, csr, "raise", settings)                          # compile, warm
            tick = time.perf_counter()
            u, flagged = vt.tree_sum(*args_, csr, "raise", settings)
            key = f"t{int(round(theta * 100))}"
            out[key], out[key + "_s"], out[key + "_flag"] = u, np.array(time.perf_counter() - tick), np.array(flagged)
            out[key + "_mean_far"] = np.array(vt.TreeStatistics.last["mean_far_nodes"])
        save(name, **out)
    if args.only in ("c2_sheet.npz", "c2_rotor.npz"):
        return

    if args.only == "network.npz" or args.only is None:
        from openfawe.aero import network_numba as nn
        out = {}
        for seed in (1, 2):
            nodes, edges, first = network_cases(seed)
            for f in (first, 0, len(nodes)):
                got = nn.incident_pairs(nodes, edges, f)
                assert np.array_equal(got, nn.incident_pairs_reference(nodes, edges, f))
                out[f"n{seed}_f{f}_pairs"] = got
            out[f"n{seed}_nodes"], out[f"n{seed}_edges"], out[f"n{seed}_first"] = nodes, edges, np.array(first)
        for name, (count, pairs) in exclusion_cases(3).items():
            ptr, seg = vn.exclusion_csr(count, pairs)
            out[f"x{name}_count"], out[f"x{name}_pairs"] = np.array(count), np.asarray(pairs, dtype=np.int64)
            out[f"x{name}_ptr"], out[f"x{name}_seg"] = ptr, seg
        save("network.npz", **out)
        if args.only:
            return

    # 1. welib per-core velocities (tests/fixtures/upstream-kernel-check.json of the reference), as arrays.
    with open(os.path.join(args.reference, "tests/fixtures/upstream-kernel-check.json"), encoding="utf-8") as f:
        data = json.load(f)
    rows = data["direct_reference_results"]
    save("upstream_kernel.npz", point=np.array([r["point"] for r in rows], dtype=np.float64),
         model=np.array([r["core_model_id"] for r in rows], dtype=np.int64),
         radius=np.array([r["core_radius_m"] for r in rows], dtype=np.float64),
         velocity=np.array([r["velocity_m_per_s"] for r in rows], dtype=np.float64),
         start=np.array(data["segment_start"], dtype=np.float64), end=np.array(data["segment_end"], dtype=np.float64))

    # 2. numba direct_sum on random networks, every core model, scalar and per-segment cores.
    out = {}
    for seed in (3, 4):
        nodes, edges, gamma, radius, points = random_network(seed)
        starts, directions, lengths = segment_arrays(nodes, edges)
        csr = vn.exclusion_csr(len(points), np.zeros((0, 2), dtype=np.int64))
        out[f"s{seed}_points"], out[f"s{seed}_starts"] = points, starts
        out[f"s{seed}_directions"], out[f"s{seed}_lengths"], out[f"s{seed}_gamma"] = directions, lengths, gamma
        out[f"s{seed}_radius"] = radius
        for model in range(6):
            for ci, core in enumerate((0.0, 0.2, radius)):
                r = np.broadcast_to(np.asarray(core, dtype=np.float64), (len(edges),)).copy()
                for sing in ("zero", "raise"):
                    u, flagged = vn.direct_sum(points, starts, directions, lengths, gamma, r, model, csr, sing)
                    key = f"s{seed}_m{model}_c{ci}_{sing}"
                    out[key] = u
                    out[key + "_flag"] = np.array(flagged)
    save("direct_random.npz", **out)

    # 3. exclusions at the network's own nodes, incident segments + random extras + duplicates.
    nodes, edges, gamma, radius, _ = random_network(5)
    starts, directions, lengths = segment_arrays(nodes, edges)
    incident = [(n, s) for s, (a, b) in enumerate(edges) for n in (a, b)]
    rng = np.random.default_rng(9)
    extra = [(int(p), int(s)) for p, s in zip(rng.integers(0, len(nodes), 30), rng.integers(0, len(edges), 30))]
    pairs = np.asarray(incident + extra + incident[:5], dtype=np.int64)
    ptr, seg = vn.exclusion_csr(len(nodes), pairs)
    out = dict(points=nodes, starts=starts, directions=directions, lengths=lengths, gamma=gamma, radius=radius,
               pairs=pairs, ptr=ptr, seg=seg)
    for model in (0, 2, 5):
        u, flagged = vn.direct_sum(nodes, starts, directions, lengths, gamma, radius, model, (ptr, seg), "raise")
        out[f"m{model}"], out[f"m{model}_flag"] = u, np.array(flagged)
    save("direct_exclusions.npz", **out)

    # 4. flag cases: on-segment point (both circulations), float-range overflow, subnormal cores.
    out = {}
    seg_nodes = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    st, di, le = segment_arrays(seg_nodes, np.array([[0, 1]]))
    cases = [("singular_g1", np.array([[0.3, 0.0, 0.0]]), st, di, le, 1.0, 0, 0.0),
             ("singular_g0", np.array([[0.3, 0.0, 0.0]]), st, di, le, 0.0, 0, 0.0)]
    tiny_nodes = np.array([[0.0, 0.0, 0.0], [1e-160, 0.0, 0.0]])
    ts, td, tl = segment_arrays(tiny_nodes, np.array([[0, 1]]))
    cases.append(("overflow", np.array([[0.0, 1e160, 0.0]]), ts, td, tl, 1.0, 0, 0.0))
    for model in (1, 2, 3):
        cases.append((f"subnormal_core_m{model}", np.array([[0.5, 1.0, 0.0]]), st, di, le, 1.0, model, 1e-310))
    for name, p, s, d, length, g, model, core in cases:
        for sing in ("raise", "zero"):
            u, flags = None, None
            u = np.zeros((1, 3))
            flags = np.zeros(1, dtype=np.int8)
            vn.sum_segments_serial(p, s, d, length, np.array([g]), np.array([core]), model, sing == "raise",
                                   np.zeros(2, dtype=np.int64), np.zeros(1, dtype=np.int64), u, flags)
            out[f"{name}_{sing}_u"], out[f"{name}_{sing}_flags"] = u, flags
            out[f"{name}_points"], out[f"{name}_starts"], out[f"{name}_directions"] = p, s, d
            out[f"{name}_lengths"], out[f"{name}_gamma"] = length, np.array([g])
            out[f"{name}_radius"], out[f"{name}_model"] = np.array([core]), np.array(model)
    save("direct_flags.npz", **out)

    # 5. config-1 lattice (16 x 128, Rosenhead-Moore) direct sum.
    case = wakes.lattice()
    csr = vn.exclusion_csr(len(case["points"]), np.zeros((0, 2), dtype=np.int64))
    u, flagged = vn.direct_sum(*wakes.backend_args(case), csr, "raise")
    save("direct_lattice.npz", u=u, flag=np.array(flagged), points_sum=np.array(case["points"].sum()),
         starts_sum=np.array(case["starts"].sum()), gamma_sum=np.array(case["gamma"].sum()))

    # 6. tree sums on the ring lattice: theta x order sweep, plus the tree and node quantities of one setting.
    nodes, edges, gamma = ring_lattice()
    rng = np.random.default_rng(2)
    points = nodes + 0.07 * rng.normal(size=nodes.shape)
    starts, directions, lengths = segment_arrays(nodes, edges)
    radius = np.full(len(edges), 0.1)
    csr = vn.exclusion_csr(len(points), np.zeros((0, 2), dtype=np.int64))
    out = dict(points=points, starts=starts, directions=directions, lengths=lengths, gamma=gamma, radius=radius)
    out["direct"], _ = vn.direct_sum(points, starts, directions, lengths, gamma, radius, 2, csr, "raise")
    for order in (0, 1, 2):
        for theta in (0.6, 0.4, 0.25, 0.15):
            settings = type("S", (), dict(theta=theta, order=order, leaf_size=8, core_clearance=3.0))()
            u, flagged = vt.tree_sum(points, starts, directions, lengths, gamma, radius, 2, csr, "raise", settings)
            out[f"o{order}_t{int(theta * 100)}"] = u
            out[f"o{order}_t{int(theta * 100)}_far"] = np.array(vt.TreeStatistics.last["mean_far_nodes"])
    lv = directions * lengths[:, None]
    ends = starts + lv
    alpha = gamma[:, None] * lv
    mid = 0.5 * (starts + ends)
    order_, lo, hi, left, right, count = vt.build_tree(mid, 8)
    centre, bound, core, m0, m1, m2 = vt.node_moments(order_, lo, hi, starts, ends, alpha, lv, radius, gamma)
    w1, t2, w2 = vt.node_contractions(m1, m2)
    out.update(order=order_, lo=lo, hi=hi, left=left, right=right, centre=centre, bound=bound, core=core, m0=m0, m1=m1,
               m2=m2, w1=w1, t2=t2, w2=w2)
    save("tree_lattice.npz", **out)

    # 7. the self-test sheet (40 rows) through tree_sum at theta 0.2 and 0.5 with exclusions, and the direct sum.
    case = wakes.selftest_sheet(40, seed=40)
    p = case["points"]
    rng = np.random.default_rng(40)
    ex = np.column_stack((rng.integers(0, len(p), 300), rng.integers(0, len(case["starts"]), 300))).astype(np.int64)
    ex = np.vstack([ex, [[0, 0], [0, 1], [5, 200]]])
    csr = vn.exclusion_csr(len(p), ex)
    out = dict(points=p, starts=case["starts"], directions=case["directions"], lengths=case["lengths"],
               gamma=case["gamma"], radius=case["radius"], pairs=ex, ptr=csr[0], seg=csr[1])
    args_ = wakes.backend_args(case)
    out["direct"], _ = vn.direct_sum(*args_, csr, "raise")
    for theta in (0.2, 0.5):
        settings = type("S", (), dict(theta=theta, order=2, leaf_size=32, core_clearance=3.0))()
        u, flagged = vt.tree_sum(*args_, csr, "raise", settings)
        out[f"t{int(theta * 100)}"] = u
        out[f"t{int(theta * 100)}_flag"] = np.array(flagged)
    save("tree_selftest.npz", **out)

    # 8. build_tree arrays on the midpoint cases of the reference's GPU-build test (tests/test_cuda_build.py:20-28).
    rng = np.random.default_rng(11)
    grid = np.array([[i * 0.5, j * 0.25, 0.0] for i in range(30) for j in range(20)])
    mids = [("random", rng.random((600, 3)) * [20.0, 5.0, 2.0], 8), ("grid", grid, 32), ("grid_leaf1", grid[:200], 1),
            ("coincident", np.ones((40, 3)), 4), ("fewer", rng.random((5, 3)), 32),
            ("long", rng.random((2100, 3)) * [30.0, 3.0, 1.0], 16)]
    out = {}
    for name, mid_, leaf in mids:
        order_, lo, hi, left, right, count = vt.build_tree(mid_, leaf)
        out.update({f"{name}_mid": mid_, f"{name}_leaf": np.array(leaf), f"{name}_order": order_, f"{name}_lo": lo,
                    f"{name}_hi": hi, f"{name}_left": left, f"{name}_right": right})
    save("tree_build.npz", **out)

    # 9. far-field forms on random symmetric moments (tests/test_vortex_tree.py:170-187 of the reference).
    rng = np.random.default_rng(5)
    count = 7
    m0 = rng.normal(size=(count, 3))
    m1 = rng.normal(size=(count, 3, 3))
    m2 = rng.normal(size=(count, 3, 3, 3))
    m2 = 0.5 * (m2 + m2.transpose(0, 1, 3, 2))
    w1, t2, w2 = vt.node_contractions(m1, m2)
    r = rng.normal(size=(count, 3, 3)) * 3.0
    far = np.zeros((count, 3, 3))
    explicit = np.zeros((count, 3, 3))
    for node in range(count):
        for order in range(3):
            far[node, order] = vt.far_velocity(*r[node, order], node, m0, m1, m2, w1, t2, w2, order)
            vt.multipole_velocity_explicit(*r[node, order], node, m0, m1, m2, order, explicit[node, order])
    save("far_field.npz", m0=m0, m1=m1, m2=m2, w1=w1, t2=t2, w2=w2, r=r, far=far, explicit=explicit)

    # 10. node moments of random segments (tests/test_cuda_moments.py:22-46 of the reference) for leaves 8, 32, 1.
    out = {}
    for seed, leaf, count in ((1, 8, 300), (2, 32, 300), (3, 1, 120)):
        rng = np.random.default_rng(seed)
        starts = rng.random((count, 3)) * [20.0, 5.0, 2.0]
        d = rng.normal(size=(count, 3))
        directions = d / np.linalg.norm(d, axis=1)[:, None]
        lengths = 0.2 + 0.3 * rng.random(count)
        gamma = rng.normal(size=count)
        gamma[::7] = 0.0
        radius = rng.uniform(0.0, 0.08, count)
        lv = directions * lengths[:, None]
        ends = starts + lv
        alpha = gamma[:, None] * lv
        order_, lo, hi, left, right, _ = vt.build_tree(0.5 * (starts + ends), leaf)
        q = vt.node_moments(order_, lo, hi, starts, ends, alpha, lv, radius, gamma)
        c = vt.node_contractions(q[4], q[5])
        pre = f"s{seed}_"
        out.update({pre + "starts": starts, pre + "directions": directions, pre + "lengths": lengths,
                    pre + "gamma": gamma, pre + "radius": radius, pre + "leaf": np.array(leaf), pre + "order": order_,
                    pre + "lo": lo, pre + "hi": hi, pre + "left": left, pre + "right": right})
        for name, value in zip(("centre", "bound", "core", "m0", "m1", "m2", "w1", "t2", "w2"), (*q, *c)):
            out[pre + name] = value
    save("moments.npz", **out)


if __name__ == "__main__":
    main()
