"""Free-wake geometry convection with every integrator stage on the device.

The reference advances the free nodes of its wake network (wake.convect_geometry, src/openfawe/aero/wake.py:535-611)
with explicit Euler, Heun or RK4 on a frozen circulation graph; each stage (``_network_convection``, wake.py:404-491)
rebuilds the incident-endpoint exclusions from the stage positions (network_numba.incident_pairs), forms the
segments from the nodes as ``segments_velocity`` does (vortex.py:460-465: starts, hypot-chained lengths, unit
directions), sums the induced velocity at the free nodes and adds the ambient flow.  Here all of that stays in HBM
between stages: exclusions by ``bs_incident_pairs`` / ``bs_exclusion_csr``, segments by tensor ops, the sum by the
direct kernel or the tree code, and the stage combinations in place.  The host sees the geometry only at the end.

Covered: the wing rows, a fixed (or linearly moving) bound row, a constant or callable ambient field, and the stage's
ring and far-wake options (``stage_parts``): rotor-ring nodes after the rows (targets with the 'zero' singularity and
their own cores), only the leading ring nodes free, the far-wake row limit with the frozen rows at the ambient flow or
drifting with the rings' induction.  The reference's surface guard stays with the caller.
"""
import numpy as np
import torch

from . import engine, network

INTEGRATORS = ("euler", "heun", "rk4")


def segments_of(nodes, edges):
    """(starts, unit directions, lengths) of the directed edges, formed as segments_velocity forms them."""
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = torch.hypot(torch.hypot(delta[:, 0], delta[:, 1]), delta[:, 2])
    if bool((lengths == 0).any()):
        raise ValueError("zero-length segment")
    return starts, delta / lengths[:, None], lengths


def _ambient(ambient, points, time):
    if callable(ambient):
        v = ambient(points, float(time))
        v = torch.as_tensor(v, dtype=torch.float64, device=points.device)
    else:
        v = torch.as_tensor(np.asarray(ambient, dtype=np.float64), device=points.device)
    return v.expand(points.shape[0], 3) if v.dim() == 1 else v


def stage_parts(n, first, node_count, edges, pairs, radii, ring_first=None, ring_free=None, ring_radii=None,
                free_rows=None, frozen_drift="ambient"):
    """The induced-velocity sums of one stage of ``_network_convection`` (wake.py:404-491) for the free nodes
    points = nodes[first:] (n of them), as a list of (lo, hi, edge_subset, cores, singularity, excluded): the velocity
    at points[lo:hi] induced by the edges edge_subset (an index tensor, or None for all) with per-edge cores ``cores``,
    under ``singularity`` (None: the caller's rule; 'zero' for ring targets), with the (point - lo, edge position in
    the subset) pairs ``excluded``.  ``pairs`` are the stage's incident (point, edge) pairs, ``radii`` and
    ``ring_radii`` per-edge cores (``ring_radii``, when given, for the ring targets only).  The wing rows are
    points[:ring_first - first], the ring nodes the rest; ``ring_free`` leading ring nodes take the induced velocity
    (None: all); with ``free_rows`` (the reference's ``free_convection_rows``) only the newest free_rows * first row
    nodes do, and with ``frozen_drift`` 'ambient_rings' the frozen rows take the induction of the ring edges (both
    nodes ring nodes).  Points in no part keep the ambient velocity.  Index arithmetic only (torch tensors on any
    device), so that the plan can be checked on the CPU."""
    rows_end = n if ring_first is None or ring_first >= node_count else ring_first - first
    ring_end = n if ring_free is None else min(n, rows_end + int(ring_free))
    target_radii = radii if ring_radii is None else ring_radii

    def shifted(lo, hi):
        keep = (pairs[:, 0] >= lo) & (pairs[:, 0] < hi)
        return pairs[keep] - torch.tensor([lo, 0], dtype=pairs.dtype, device=pairs.device)

    parts = []
    if free_rows is not None and int(free_rows) * first < rows_end:
        free = int(free_rows) * first
        parts.append((0, free, None, radii, None, shifted(0, free)))
        if frozen_drift == "ambient_rings" and ring_first is not None and ring_first < node_count:
            ring_edge = (edges >= ring_first).all(dim=1)
            if bool(ring_edge.any()):
                sub = torch.nonzero(ring_edge).reshape(-1)
                remap = torch.full((edges.shape[0],), -1, dtype=pairs.dtype, device=pairs.device)
                remap[sub] = torch.arange(sub.numel(), dtype=pairs.dtype, device=pairs.device)
                frozen = shifted(free, rows_end)
                frozen = frozen[ring_edge[frozen[:, 1]]]
                frozen = torch.stack((frozen[:, 0], remap[frozen[:, 1]]), dim=1)
                parts.append((free, rows_end, sub, radii[sub], None, frozen))
        if rows_end < ring_end:
            parts.append((rows_end, ring_end, None, target_radii, "zero", shifted(rows_end, ring_end)))
    elif ring_first is None or ring_first >= node_count:
        parts.append((0, n, None, radii, None, pairs))
    else:
        split = ring_first - first
        parts.append((0, split, None, radii, None, shifted(0, split)))
        if split < ring_end:
            parts.append((split, ring_end, None, target_radii, "zero", shifted(split, ring_end)))
    return parts


def network_velocity(nodes, edges, gamma, radii, first, model, ambient=(0.0, 0.0, 0.0), time=0.0, method="tree",
                     precision="mixed", singularity="raise", theta=0.1, order=3, leaf_size=32, block=128, near=3.0,
                     ring_first=None, ring_free=None, ring_radii=None, free_rows=None, frozen_drift="ambient"):
    """Velocity [n - first, 3] (device tensor) of the free nodes nodes[first:]: ambient plus the induced velocity of
    the network, with every free node excluded from the segments ending at its position (one stage of
    ``_network_convection``; the ring and far-wake options as in ``stage_parts``, per-edge ``radii`` and
    ``ring_radii``)."""
    dev = nodes.device
    points = nodes[first:]
    velocity = _ambient(ambient, points, time).clone()
    if edges.shape[0] == 0 or points.shape[0] == 0:
        return velocity
    def per_edge(cores):
        cores = engine.f64(cores, dev).reshape(-1)
        return cores.expand(edges.shape[0]).contiguous() if cores.numel() == 1 else cores

    radii = per_edge(radii)
    ring_radii = None if ring_radii is None else per_edge(ring_radii)
    pairs = network.incident_pairs_device(nodes, edges, first)
    parts = stage_parts(points.shape[0], first, nodes.shape[0], edges, pairs, radii, ring_first, ring_free,
                        ring_radii, free_rows, frozen_drift)
    starts, directions, lengths = segments_of(nodes, edges)
    for lo, hi, sub, cores, rule, excluded in parts:
        if hi <= lo:
            continue
        rule = rule or singularity
        csr = network.exclusion_csr_device(hi - lo, excluded)
        if sub is None:
            src = engine.Sources(starts, directions, lengths, gamma, cores, dev)
        else:
            src = engine.Sources(starts[sub], directions[sub], lengths[sub], gamma[sub], cores, dev)
        tgt = engine.Targets(points[lo:hi], csr if csr[1].numel() else None, dev)
        if method == "direct":
            u, flags = engine.direct(src, tgt, model, rule, precision, block, near)
        elif method == "tree":
            u, flags, _ = engine.tree_sum(src, tgt, model, rule, precision, block, near, theta, order, leaf_size,
                                          3.0, "morton", far_counts=False)
        else:
            raise ValueError("method must be 'direct' or 'tree'")
        if bool(flags.any()):
            raise RuntimeError("a free node lies on a filament of the wake (the reference raises for this pair)")
        if not bool(torch.isfinite(u).all()):
            raise ValueError("velocity exceeds finite float64 range")
        velocity[lo:hi] += u
    return velocity


def convect(nodes, edges, gamma, radii, first, model, dt, ambient=(0.0, 0.0, 0.0), integrator="rk4", substeps=1,
            time=0.0, next_bound=None, drift=None, **options):
    """Advance the free nodes nodes[first:] by dt (substeps explicit steps of the integrator) on the frozen graph;
    returns their new positions (device tensor [n - first, 3]).  The bound nodes nodes[:first] stay put, or move
    linearly to ``next_bound`` over the step (the reference's stage interpolation).  ``drift`` ([n - first, 3], or
    None) is added to every stage's velocity, as the reference adds its frozen rings' sheet drift (wake.py:584-592).
    ``options`` go to ``network_velocity`` (method, precision, theta, order, the ring and far-wake options)."""
    if integrator not in INTEGRATORS:
        raise ValueError(f"integrator must be one of {INTEGRATORS}")
    dev = nodes.device if isinstance(nodes, torch.Tensor) else engine._device_of(options.pop("device", None))
    nodes = engine.f64(nodes, dev).reshape(-1, 3)
    edges = engine.i64(edges, dev).reshape(-1, 2)
    gamma = engine.f64(gamma, dev).reshape(-1)
    radii = engine.f64(radii, dev).reshape(-1)
    if radii.numel() == 1:
        radii = radii.expand(edges.shape[0]).contiguous()
    bound = nodes[:first]
    displacement = None if next_bound is None else engine.f64(next_bound, dev).reshape(-1, 3) - bound
    drift = None if drift is None else engine.f64(drift, dev).reshape(-1, 3)
    points = nodes[first:].clone()
    h = float(dt) / int(substeps)
    t0 = float(time)

    def rhs(current, t):
        stage_bound = bound if displacement is None or t == t0 else bound + ((t - t0) / float(dt)) * displacement
        velocity = network_velocity(torch.cat((stage_bound, current)), edges, gamma, radii, first, model, ambient, t,
                                    **options)
        return velocity if drift is None else velocity + drift

    for k in range(int(substeps)):
        t = t0 + k * h
        k1 = rhs(points, t)
        if integrator == "euler":
            points = points + h * k1
        elif integrator == "heun":
            k2 = rhs(points + h * k1, t + h)
            points = points + h * (k1 + k2) / 2
        else:
            k2 = rhs(points + h * k1 / 2, t + h / 2)
            k3 = rhs(points + h * k2 / 2, t + h / 2)
            k4 = rhs(points + h * k3, t + h)
            points = points + h * (k1 + 2 * k2 + 2 * k3 + k4) / 6
    return points
