"""Convection stages and frozen wake states.

CPU: the oracle's composition of the reference's stage (incident pairs -> exclusion CSR -> segments formed as
segments_velocity forms them -> ordered FP64 direct sum, plus the ambient flow) reproduces the reference's
``_network_convection`` velocities and Euler / Heun / RK4 steps bit for bit (fixtures made by the reference's own code),
and a saved frozen state reloads to the same arrays and the reference's ``segments_velocity`` result.
GPU: the device-resident convection and the loaded state on the device, against the same fixtures: FP64 direct within
the reference's A1 bound (1e-12 * sum_s |u_s| per point, and that bound times dt for a step), the mixed tree within
1e-5 relative L2 of the step's displacement.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden
from oracle import oracle as O


def oracle_stage(nodes, edges, gamma, radii, first, model, inflow):
    """wake._network_convection for a network without rings, restated with the oracle (test infrastructure)."""
    points = nodes[first:]
    pairs = O.incident_pairs(nodes, edges, first)
    csr = O.exclusion_csr(len(points), pairs)
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
    u, flag = O.direct_sum(points, starts, delta / lengths[:, None], lengths, gamma, radii, model, csr, "raise")
    assert not flag
    velocity = np.broadcast_to(inflow, points.shape).copy()
    velocity += u
    return velocity


def oracle_step(g, integrator):
    nodes, edges, gamma, radii, first = g["nodes"], g["edges"], g["gamma"], g["radii"], int(g["first"])
    inflow, dt = g["inflow"], float(g["dt"])

    def rhs(points):
        return oracle_stage(np.concatenate((nodes[:first], points)), edges, gamma, radii, first, 2, inflow)
    points = nodes[first:].copy()
    k1 = rhs(points)
    if integrator == "euler":
        return points + dt * k1
    if integrator == "heun":
        return points + dt * (k1 + rhs(points + dt * k1)) / 2
    k2 = rhs(points + dt * k1 / 2)
    k3 = rhs(points + dt * k2 / 2)
    k4 = rhs(points + dt * k3)
    return points + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6


def test_oracle_convection_stages_match_reference():
    g = golden("convection.npz")
    k1 = oracle_stage(g["nodes"], g["edges"], g["gamma"], g["radii"], int(g["first"]), 2, g["inflow"])
    assert np.array_equal(k1.view(np.uint64), g["k1"].view(np.uint64))
    for integrator in ("euler", "heun", "rk4"):
        got = oracle_step(g, integrator)
        assert np.array_equal(got.view(np.uint64), g[integrator].view(np.uint64)), integrator


# the five settings of convection_rings.npz (tests/golden/make_golden.py)
RING_SETTINGS = {"rings": {}, "ring_free": {"ring_free": 200, "ring_radii": True},
                 "row_limit": {"free_rows": 3, "frozen_drift": "ambient"},
                 "row_limit_rings": {"free_rows": 3, "frozen_drift": "ambient_rings"},
                 "all": {"ring_free": 200, "ring_radii": True, "free_rows": 3, "frozen_drift": "ambient_rings"}}


def ring_options(g, name, to_tensor):
    opt = dict(RING_SETTINGS[name])
    opt["ring_radii"] = to_tensor(g["ring_radii"]) if opt.get("ring_radii") else None
    return dict(ring_first=int(g["ring_first"]), **opt)


def oracle_ring_stage(g, name, nodes=None):
    """One stage of wake._network_convection with rotor rings: the sums convection.stage_parts plans, each by the
    oracle's ordered FP64 direct sum, added to the ambient flow (test infrastructure)."""
    import torch
    from openfawe_b200 import convection
    nodes = g["nodes"] if nodes is None else nodes
    edges, gamma, radii = g["edges"], g["gamma"], g["radii"]
    first = int(g["first"])
    points = nodes[first:]
    pairs = O.incident_pairs(nodes, edges, first)
    parts = convection.stage_parts(len(points), first, len(nodes), torch.as_tensor(edges), torch.as_tensor(pairs),
                                   torch.as_tensor(radii), **ring_options(g, name, torch.as_tensor))
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
    directions = delta / lengths[:, None]
    velocity = np.broadcast_to(g["inflow"], points.shape).copy()
    for lo, hi, sub, cores, rule, excluded in parts:
        take = slice(None) if sub is None else sub.numpy()
        csr = O.exclusion_csr(hi - lo, excluded.numpy())
        u, flag = O.direct_sum(points[lo:hi], starts[take], directions[take], lengths[take], gamma[take],
                               cores.numpy(), 2, csr, rule or "raise")
        assert not flag
        velocity[lo:hi] += u
    return velocity


def test_oracle_ring_stages_match_reference():
    """Rows and rings, the leading ring nodes free with their own cores, the far-wake row limit with frozen rows at
    the ambient flow or drifting with the rings: the planned sums reproduce the reference's stage bit for bit."""
    g = golden("convection_rings.npz")
    for name in RING_SETTINGS:
        got = oracle_ring_stage(g, name)
        assert np.array_equal(got.view(np.uint64), g[name].view(np.uint64)), name


def test_stage_plan_edge_cases():
    """The plan's edge cases, by the reference's rules (wake.py:431-491): ring_first past the last node is a network
    without rings; ring_free 0 leaves every ring node at the ambient flow; a row limit that covers every row is no
    limit; no ring edge means no frozen-row drift."""
    import torch
    from openfawe_b200 import convection
    g = golden("convection_rings.npz")
    nodes, edges, radii = g["nodes"], torch.as_tensor(g["edges"]), torch.as_tensor(g["radii"])
    first, ring_first = int(g["first"]), int(g["ring_first"])
    n = len(nodes) - first
    pairs = torch.as_tensor(O.incident_pairs(nodes, g["edges"], first))
    plan = lambda **kw: convection.stage_parts(n, first, len(nodes), edges, pairs, radii, **kw)  # noqa: E731
    spans = lambda parts: [(lo, hi, rule) for lo, hi, _, _, rule, _ in parts]  # noqa: E731
    assert spans(plan(ring_first=len(nodes))) == spans(plan()) == [(0, n, None)]
    assert spans(plan(ring_first=ring_first, ring_free=0)) == [(0, ring_first - first, None)]
    rows = ring_first - first
    assert spans(plan(ring_first=ring_first, free_rows=rows // first + 1)) == \
        [(0, rows, None), (rows, n, "zero")]
    no_rings = plan(free_rows=2, frozen_drift="ambient_rings")
    assert spans(no_rings) == [(0, 2 * first, None)]
    # every planned exclusion names a point of its part and an edge of its subset
    for lo, hi, sub, cores, rule, excluded in plan(ring_first=ring_first, free_rows=3, frozen_drift="ambient_rings"):
        width = len(edges) if sub is None else len(sub)
        assert len(cores) == width
        if len(excluded):
            assert int(excluded[:, 0].min()) >= 0 and int(excluded[:, 0].max()) < hi - lo
            assert int(excluded[:, 1].min()) >= 0 and int(excluded[:, 1].max()) < width


def test_frozen_state_roundtrip_and_oracle(tmp_path):
    from openfawe_b200 import wakestate
    state = wakestate.load_state(os.path.join(GOLDEN, "frozen_state_input.npz"))
    path = str(tmp_path / "state_0001.npz")
    wakestate.save_state(path, state["nodes"], state["edges"], state["gamma"], state["radii"], state["first"],
                         state["speed"], state["core_model"], state["exclusions"])
    again = wakestate.load_state(path)
    for key in wakestate.KEYS:
        assert np.array_equal(np.asarray(again[key]), np.asarray(state[key])), key
    nodes, edges, first = state["nodes"], state["edges"], state["first"]
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
    csr = O.exclusion_csr(len(nodes) - first, state["exclusions"])
    u, _ = O.direct_sum(nodes[first:], starts, delta / lengths[:, None], lengths, state["gamma"], state["radii"], 2,
                        csr, "raise")
    assert np.array_equal(u.view(np.uint64), golden("frozen_state.npz")["u"].view(np.uint64))
    with pytest.raises(ValueError):
        np.savez(str(tmp_path / "bad.npz"), nodes=nodes)
        wakestate.load_state(str(tmp_path / "bad.npz"))


def _a1_scale(nodes, edges, gamma, radii, first):
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
    pairs, _ = O.pair_matrix(nodes[first:], starts, delta / lengths[:, None], lengths, radii, 2, False)
    return (np.linalg.norm(pairs, axis=2) * np.abs(gamma)[None, :]).sum(axis=1)


@pytest.mark.gpu
def test_device_convection_matches_reference_steps(device):
    from openfawe_b200 import convection
    g = golden("convection.npz")
    nodes, edges, gamma, radii, first = g["nodes"], g["edges"], g["gamma"], g["radii"], int(g["first"])
    dt = float(g["dt"])
    scale = _a1_scale(nodes, edges, gamma, radii, first)
    import torch
    dnodes = torch.as_tensor(nodes, device=device)
    v = convection.network_velocity(dnodes, torch.as_tensor(edges, device=device), torch.as_tensor(gamma, device=device),
                                    torch.as_tensor(radii, device=device), first, 2, g["inflow"], method="direct",
                                    precision="fp64")
    err = np.linalg.norm(v.cpu().numpy() - g["k1"], axis=1)
    assert np.all(err <= 1e-12 * scale), float((err / scale).max())
    for integrator in ("euler", "heun", "rk4"):
        got = convection.convect(nodes, edges, gamma, radii, first, 2, dt, g["inflow"], integrator, method="direct",
                                 precision="fp64", device=device).cpu().numpy()
        err = np.linalg.norm(got - g[integrator], axis=1)
        assert np.all(err <= 4e-12 * scale * dt + 1e-15), integrator
        step = g[integrator] - nodes[first:]
        tree = convection.convect(nodes, edges, gamma, radii, first, 2, dt, g["inflow"], integrator, method="tree",
                                  precision="mixed", theta=0.1, order=3, device=device).cpu().numpy()
        assert np.linalg.norm(tree - g[integrator]) / np.linalg.norm(step) < 1e-5, integrator


@pytest.mark.gpu
def test_device_ring_stages_match_reference(device):
    """The device stage with the ring and far-wake options, FP64 direct sums, within the A1 bound of the reference's."""
    import torch
    from openfawe_b200 import convection
    g = golden("convection_rings.npz")
    nodes, edges, gamma, radii, first = g["nodes"], g["edges"], g["gamma"], g["radii"], int(g["first"])
    scale = _a1_scale(nodes, edges, gamma, np.maximum(radii, g["ring_radii"]), first)
    dev = lambda a: torch.as_tensor(a, device=device)  # noqa: E731
    for name in RING_SETTINGS:
        v = convection.network_velocity(dev(nodes), dev(edges), dev(gamma), dev(radii), first, 2, g["inflow"],
                                        method="direct", precision="fp64", **ring_options(g, name, dev))
        err = np.linalg.norm(v.cpu().numpy() - g[name], axis=1)
        assert np.all(err <= 1e-12 * scale), (name, float((err / scale).max()))


@pytest.mark.gpu
def test_device_ring_rk4_step_with_drift(device):
    """An RK4 step with the ring and far-wake options and a constant drift of the frozen ring nodes (the reference's
    sheet drift): the device step against the oracle's composition of the planned stages (itself pinned stage by stage
    and integrator by integrator to the reference), within the A1 bound times dt."""
    from openfawe_b200 import convection
    g = golden("convection_rings.npz")
    name = "ring_free"
    nodes, edges, gamma, radii, first = g["nodes"], g["edges"], g["gamma"], g["radii"], int(g["first"])
    dt = 0.02
    drift = np.zeros((len(nodes) - first, 3))
    drift[int(g["ring_first"]) - first + 200:] = [0.4, -0.1, 0.2]

    def rhs(points):
        return oracle_ring_stage(g, name, np.concatenate((nodes[:first], points))) + drift
    points = nodes[first:]
    k1 = rhs(points)
    k2 = rhs(points + dt * k1 / 2)
    k3 = rhs(points + dt * k2 / 2)
    k4 = rhs(points + dt * k3)
    want = points + dt * (k1 + 2 * k2 + 2 * k3 + k4) / 6
    import torch
    got = convection.convect(nodes, edges, gamma, radii, first, 2, dt, g["inflow"], "rk4", method="direct",
                             precision="fp64", device=device, drift=drift,
                             **ring_options(g, name, lambda a: torch.as_tensor(a, device=device))).cpu().numpy()
    scale = _a1_scale(nodes, edges, gamma, np.maximum(radii, g["ring_radii"]), first)
    err = np.linalg.norm(got - want, axis=1)
    assert np.all(err <= 4e-12 * scale * dt + 1e-15), float((err / (scale * dt)).max())
    moved = np.linalg.norm(got - points, axis=1)
    assert np.all(moved > 0)


@pytest.mark.gpu
def test_frozen_state_on_device(device):
    from openfawe_b200 import wakestate
    wake = wakestate.FrozenWake(os.path.join(GOLDEN, "frozen_state_input.npz"), device)
    ref = golden("frozen_state.npz")["u"]
    s = wake.state
    scale = _a1_scale(s["nodes"], s["edges"], s["gamma"], s["radii"], s["first"])
    # excluded pairs are left out of the reference's sum, so the bound uses the full scale (larger, still tight)
    u, flags = wake.velocity("direct", "fp64")
    assert not flags.any()
    assert np.all(np.linalg.norm(u.cpu().numpy() - ref, axis=1) <= 1e-12 * scale)
    ut, _ = wake.velocity("tree", "mixed", theta=0.1, order=3)
    assert np.linalg.norm(ut.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-5
    assert wake.error_over_speed(ut, ref) < 1e-4
