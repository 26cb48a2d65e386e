"""The CPU oracle pinned against the reference's own outputs (tests/golden/, made by running the reference's numba code).

The oracle (oracle/bs_oracle.c) restates vortex_numba.pair_velocity / direct_sum and vortex_tree.build_tree /
node_moments / far_velocity / tree_velocity operation for operation; these checks require bit-for-bit equality with
the reference wherever the reference's arithmetic is deterministic (everything here), plus the reference's own
analytical known answers (tests/test_vortex.py, test_rosenhead.py, test_vortex_tree.py of the reference).
"""
import numpy as np
import pytest

from conftest import golden, no_exclusions
from oracle import oracle as O


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def seg(start, end):
    start, end = np.asarray(start, float), np.asarray(end, float)
    d = end - start
    length = np.hypot(np.hypot(d[0], d[1]), d[2])
    return start[None], (d / length)[None], np.array([length])


A, B = [0.0, 0.0, -1.0], [0.0, 0.0, 1.0]


def one(point, model=0, core=0.0, gamma=1.0, start=A, end=B, singularity="raise"):
    s, d, length = seg(start, end)
    u, flag = O.direct_sum(np.array([point], float), s, d, length, np.array([gamma]), np.array([core]), model,
                           no_exclusions(1), singularity)
    return u[0], flag


class TestKnownAnswers:
    def test_k01_closed_form(self):
        u, _ = one([1, 0, 0])
        np.testing.assert_allclose(u, [0, 1 / (2 * np.pi * np.sqrt(2)), 0], rtol=1e-12, atol=1e-14)

    def test_k02_symmetric_all_cores(self):
        for h in (0.05, 1.0, 10.0):
            ideal = 1 / (2 * np.pi * h * np.sqrt(1 + h * h))
            q = (h / 0.5) ** 2
            factors = [1, min(q, 1), 1 if -1.25643 * q < -10 else -np.expm1(-1.25643 * q), q / np.sqrt(1 + q * q),
                       (2 * h * h * (1 + h * h)) / (2 * h * h * (1 + h * h) + 4 * 0.5 ** 2),
                       h * h * np.sqrt(1 + h * h) / ((h * h + 0.5 ** 2) * np.sqrt(1 + h * h + 0.5 ** 2))]
            for model in range(6):
                u, _ = one([h, 0, 0], model, 0.5)
                np.testing.assert_allclose(u, [0, ideal * factors[model], 0], rtol=1e-12, atol=1e-14)

    def test_lamb_cutoff(self):
        for exponent in (9.99, 10.01):
            h = 0.5 * np.sqrt(exponent / 1.25643)
            ideal = 1 / (2 * np.pi * h * np.sqrt(1 + h * h))
            u, _ = one([h, 0, 0], 2, 0.5)
            expected = ideal * -np.expm1(-exponent) if exponent < 10 else ideal
            np.testing.assert_allclose(u[1], expected, rtol=1e-12, atol=1e-14)

    def test_welib_upstream_values(self):
        g = golden("upstream_kernel.npz")
        for point, model, radius, velocity in zip(g["point"], g["model"], g["radius"], g["velocity"]):
            u, _ = one(point, int(model), float(radius), start=g["start"], end=g["end"])
            np.testing.assert_allclose(u, velocity, rtol=1e-12, atol=1e-14)

    def test_gauss_legendre_quadrature(self):
        start, end, point = np.array([-0.7, 0.3, -0.8]), np.array([1.2, -0.4, 1.0]), np.array([0.5, 1.2, 0.4])
        x, w = np.polynomial.legendre.leggauss(96)
        delta = end - start
        r = point - (start + ((x + 1) / 2)[:, None] * delta)
        integral = np.sum((w / 2)[:, None] * np.cross(delta, r) / np.linalg.norm(r, axis=1)[:, None] ** 3, axis=0)
        u, _ = one(point, gamma=1.7, start=start, end=end)
        np.testing.assert_allclose(u, 1.7 / (4 * np.pi) * integral, rtol=1e-12, atol=1e-14)

    def test_near_interior_stable(self):
        h = 1e-9
        u, _ = one([h, 0, 0])
        np.testing.assert_allclose(u[1], 1 / (2 * np.pi * h * np.sqrt(1 + h * h)), rtol=1e-12)

    def test_square_ring_centre(self):
        corners = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], dtype=float)
        s = corners
        e = np.roll(corners, -1, axis=0)
        d = e - s
        length = np.hypot(np.hypot(d[:, 0], d[:, 1]), d[:, 2])
        u, _ = O.direct_sum(np.zeros((1, 3)), s, d / length[:, None], length, np.ones(4), np.zeros(4), 0,
                            no_exclusions(1), "raise")
        np.testing.assert_allclose(u[0], [0, 0, np.sqrt(2) / np.pi], rtol=1e-12, atol=1e-14)

    def test_singular_and_zero(self):
        _, flag = one([0, 0, 0])
        assert flag
        u, flag = one([0, 0, 0], singularity="zero")
        assert not flag and np.all(u == 0)
        u, flag = one([0, 0, 2])
        assert not flag and np.all(u == 0)


class TestDirectAgainstReference:
    def test_random_networks_every_model_bitwise(self):
        g = golden("direct_random.npz")
        for seed in (3, 4):
            P = lambda k: g[f"s{seed}_{k}"]  # noqa: E731
            csr = no_exclusions(len(P("points")))
            for model in range(6):
                for ci, core in enumerate((0.0, 0.2, P("radius"))):
                    r = np.broadcast_to(np.asarray(core, dtype=np.float64), (len(P("gamma")),)).copy()
                    for sing in ("zero", "raise"):
                        key = f"s{seed}_m{model}_c{ci}_{sing}"
                        u, flag = O.direct_sum(P("points"), P("starts"), P("directions"), P("lengths"), P("gamma"),
                                               r, model, csr, sing)
                        assert bits_equal(u, g[key]), key
                        assert flag == bool(g[key + "_flag"]), key

    def test_exclusions_bitwise(self):
        g = golden("direct_exclusions.npz")
        ptr, seg_ = O.exclusion_csr(len(g["points"]), g["pairs"])
        assert np.array_equal(ptr, g["ptr"]) and np.array_equal(seg_, g["seg"])
        for model in (0, 2, 5):
            u, flag = O.direct_sum(g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"],
                                   model, (ptr, seg_), "raise")
            assert bits_equal(u, g[f"m{model}"])
            assert flag == bool(g[f"m{model}_flag"])

    def test_flag_cases(self):
        g = golden("direct_flags.npz")
        names = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_points")})
        assert len(names) == 6
        for name in names:
            for sing in ("raise", "zero"):
                u, flags = O.direct_sum(g[f"{name}_points"], g[f"{name}_starts"], g[f"{name}_directions"],
                                        g[f"{name}_lengths"], g[f"{name}_gamma"], g[f"{name}_radius"],
                                        int(g[f"{name}_model"]), no_exclusions(1), sing, return_flags=True)
                assert np.array_equal(flags, g[f"{name}_{sing}_flags"]), (name, sing)
                assert bits_equal(u, g[f"{name}_{sing}_u"]), (name, sing)

    def test_lattice_config(self):
        from openfawe_b200 import wakes
        g = golden("direct_lattice.npz")
        case = wakes.lattice()
        assert case["points"].sum() == g["points_sum"] and case["starts"].sum() == g["starts_sum"]
        u, flag = O.direct_sum(*wakes.backend_args(case), no_exclusions(len(case["points"])), "raise")
        assert bits_equal(u, g["u"]) and flag == bool(g["flag"])

    def test_pair_matrix_rows_sum_to_direct(self):
        g = golden("direct_random.npz")
        P = lambda k: g[f"s3_{k}"]  # noqa: E731
        pairs, flags = O.pair_matrix(P("points"), P("starts"), P("directions"), P("lengths"), P("radius"), 2, False)
        u, _ = O.direct_sum(P("points"), P("starts"), P("directions"), P("lengths"), P("gamma"), P("radius"), 2,
                            no_exclusions(len(P("points"))), "zero")
        np.testing.assert_allclose(np.einsum("psk,s->pk", pairs, P("gamma")), u, rtol=1e-12, atol=1e-12)


class TestTreeAgainstReference:
    def test_build_tree_element_for_element(self):
        g = golden("tree_build.npz")
        for name in ("random", "grid", "grid_leaf1", "coincident", "fewer", "long"):
            order, lo, hi, left, right, _ = O.build_tree(g[f"{name}_mid"], int(g[f"{name}_leaf"]))
            for key, value in zip(("order", "lo", "hi", "left", "right"), (order, lo, hi, left, right)):
                assert np.array_equal(value, g[f"{name}_{key}"]), (name, key)

    def test_node_moments_bitwise(self):
        g = golden("moments.npz")
        for seed in (1, 2, 3):
            p = lambda k: g[f"s{seed}_{k}"]  # noqa: E731
            lv, ends, alpha, mid = O.segment_geometry(p("starts"), p("directions"), p("lengths"), p("gamma"))
            order, lo, hi, left, right, _ = O.build_tree(mid, int(p("leaf")))
            assert np.array_equal(order, p("order")) and np.array_equal(lo, p("lo"))
            q = O.node_moments(order, lo, hi, p("starts"), ends, alpha, lv, p("radius"), p("gamma"))
            c = O.node_contractions(q[4], q[5])
            for name, value in zip(("centre", "bound", "core", "m0", "m1", "m2", "w1", "t2", "w2"), (*q, *c)):
                assert bits_equal(value, p(name)), (seed, name)

    def test_far_field_forms(self):
        g = golden("far_field.npz")
        for node in range(len(g["m0"])):
            for order in range(3):
                u = O.far_velocity(g["r"][node, order], g["m0"][node], g["m1"][node], g["m2"][node], g["w1"][node],
                                   g["t2"][node], g["w2"][node], order)
                assert bits_equal(u, g["far"][node, order])
                np.testing.assert_allclose(u, g["explicit"][node, order], rtol=1e-12,
                                           atol=1e-14 * np.abs(g["explicit"][node, order]).max())

    def test_tree_sum_theta_order_sweep_bitwise(self):
        g = golden("tree_lattice.npz")
        args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2,
                no_exclusions(len(g["points"])), "raise")
        for order in (0, 1, 2):
            for theta in (0.6, 0.4, 0.25, 0.15):
                u, flag, d = O.tree_sum(*args, theta=theta, order=order, leaf_size=8, details=True)
                key = f"o{order}_t{int(theta * 100)}"
                assert bits_equal(u, g[key]), key
                assert d["far"].mean() == float(g[key + "_far"]), key
        # the reference's convergence checks (tests/test_vortex_tree.py:45-65 of the reference)
        scale = np.max(np.linalg.norm(g["direct"], axis=1))
        errors = {(o, t): np.max(np.linalg.norm(g[f"o{o}_t{int(t * 100)}"] - g["direct"], axis=1)) / scale
                  for o in (0, 1, 2) for t in (0.6, 0.4, 0.25, 0.15)}
        for o in (0, 1, 2):
            seq = [errors[o, t] for t in (0.6, 0.4, 0.25, 0.15)]
            assert all(b < a for a, b in zip(seq, seq[1:]))
        assert errors[2, 0.15] < 2e-4

    def test_selftest_sheet_with_exclusions_bitwise(self):
        g = golden("tree_selftest.npz")
        args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2,
                (g["ptr"], g["seg"]), "raise")
        u, _ = O.direct_sum(*args)
        assert bits_equal(u, g["direct"])
        for theta in (0.2, 0.5):
            u, flag = O.tree_sum(*args, theta=theta)
            assert bits_equal(u, g[f"t{int(theta * 100)}"]) and flag == bool(g[f"t{int(theta * 100)}_flag"])

    def test_tiny_theta_is_direct(self):
        g = golden("tree_lattice.npz")
        args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2,
                no_exclusions(len(g["points"])), "raise")
        u, _ = O.tree_sum(*args, theta=1e-9, leaf_size=4)
        scale = np.max(np.linalg.norm(g["direct"], axis=1))
        np.testing.assert_allclose(u, g["direct"], rtol=0, atol=1e-13 * scale)

    def test_unsupported_core_models_refused(self):
        g = golden("tree_lattice.npz")
        for model in (3, 4, 5):
            with pytest.raises(ValueError):
                O.tree_sum(g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], model,
                           no_exclusions(len(g["points"])), "raise")


class TestMortonRecomputation:
    """The CPU statement of the B200 Morton tree: structural invariants (the GPU is checked against it bit for bit)."""

    def test_tree_invariants(self):
        from openfawe_b200 import wakes
        case = wakes.selftest_sheet(30, seed=30)
        for leaf in (1, 8, 32):
            t = O.morton_tree(case["starts"], case["directions"], case["lengths"], leaf)
            m = len(case["starts"])
            assert np.array_equal(np.sort(t["order"]), np.arange(m))
            assert np.all(np.diff(t["sorted_keys"].astype(object)) >= 0)
            assert np.array_equal(t["keys"][t["order"]], t["sorted_keys"])
            lo, hi, left, right = t["lo"], t["hi"], t["left"], t["right"]
            assert lo[0] == 0 and hi[0] == m
            inner = left >= 0
            assert np.all((left >= 0) == (right >= 0))
            assert np.all(lo[left[inner]] == lo[inner]) and np.all(hi[right[inner]] == hi[inner])
            assert np.all(hi[left[inner]] == lo[right[inner]])
            assert np.all(hi[inner] - lo[inner] > leaf)
            leaves = ~inner
            assert np.all(hi[leaves] - lo[leaves] <= max(leaf, 1))
            covered = np.zeros(m, dtype=int)
            for a, b in zip(lo[leaves], hi[leaves]):
                covered[a:b] += 1
            assert np.all(covered == 1)

    def test_morton_tree_sum_converges(self):
        g = golden("tree_lattice.npz")
        args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2,
                no_exclusions(len(g["points"])), "raise")
        scale = np.max(np.linalg.norm(g["direct"], axis=1))
        previous = np.inf
        for theta in (0.6, 0.3, 0.15):
            u, _ = O.tree_sum(*args, theta=theta, leaf_size=8, kind="morton")
            error = np.max(np.linalg.norm(u - g["direct"], axis=1)) / scale
            assert error < previous
            previous = error
        u, _ = O.tree_sum(*args, theta=1e-9, leaf_size=4, kind="morton")
        np.testing.assert_allclose(u, g["direct"], rtol=0, atol=1e-13 * scale)


def test_incident_pairs_and_exclusion_csr_match_reference():
    """network_numba.incident_pairs (sorted-bits version, equal to its dictionary reference) and
    vortex_numba.exclusion_csr: bound/free coincidences, repeated free nodes, -0.0 vs 0.0, NaN, inf; first = bound
    count, 0 and n; exclusion pairs with repeats, negative and 2**62 segment ids, empty input."""
    g = golden("network.npz")
    for seed in (1, 2):
        nodes, edges, first = g[f"n{seed}_nodes"], g[f"n{seed}_edges"], int(g[f"n{seed}_first"])
        for f in (first, 0, len(nodes)):
            assert np.array_equal(O.incident_pairs(nodes, edges, f), g[f"n{seed}_f{f}_pairs"]), (seed, f)
    for name in "abcd":
        ptr, seg_ = O.exclusion_csr(int(g[f"x{name}_count"]), g[f"x{name}_pairs"])
        assert np.array_equal(ptr, g[f"x{name}_ptr"]) and np.array_equal(seg_, g[f"x{name}_seg"]), name


def test_pair_matrix_and_assemble_columns_match_reference():
    """vortex_numba.pair_matrix and assemble_columns on a 16-panel ring wing's column layout (bound line, trailing
    legs, shed rings; points on segments for the flags), models 0, 2, 5, both singularity modes: bit for bit."""
    from openfawe_b200 import wakes
    g = golden("operators.npz")
    wing = wakes.ring_wing(panels=16, rows=3)
    for model in (0, 2, 5):
        radius = wing["radius"] if model else np.zeros(len(wing["radius"]))
        for mode in ("raise", "zero"):
            key = f"m{model}_{mode}"
            pairs, flags = O.pair_matrix(g["points"], wing["starts"], wing["directions"], wing["lengths"], radius,
                                         model, mode == "raise")
            assert bits_equal(pairs, g[key + "_pairs"]) and np.array_equal(flags, g[key + "_flags"]), key
            cols = O.assemble_columns(pairs, wing["column_ptr"], wing["column_segment"], wing["column_sign"])
            assert bits_equal(cols, g[key + "_columns"]), key
