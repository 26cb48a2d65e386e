"""Free-wake geometry convection with every integrator stage on the device.

The reference advances the free nodes of its wake network (wake.convect_geometry, src/openfawe/aero/wake.py:535-611)
with explicit Euler, Heun or RK4 on a frozen circulation graph; each stage (``_network_convection``, wake.py:404-491)
rebuilds the incident-endpoint exclusions from the stage positions (network_numba.incident_pairs), forms the
segments from the nodes as ``segments_velocity`` does (vortex.py:460-465: starts, hypot-chained lengths, unit
directions), sums the induced velocity at the free nodes and adds the ambient flow.  Here all of that stays in HBM
between stages: exclusions by ``bs_incident_pairs`` / ``bs_exclusion_csr``, segments by tensor ops, the sum by the
direct kernel or the tree code, and the stage combinations in place.  The host sees the geometry only at the end.

Covered: the wing rows without rotor rings, a fixed (or linearly moving) bound row, a constant or callable ambient
field; the reference's ring bookkeeping, surface guard and far-wake row limit stay with the caller.
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


def network_velocity(nodes, edges, gamma, radii, first, model, ambient=(0.0, 0.0, 0.0), time=0.0, method="tree",
                     precision="mixed", singularity="raise", theta=0.1, order=3, leaf_size=32, block=128, near=3.0):
    """Velocity [n - first, 3] (device tensor) of the free nodes nodes[first:]: ambient plus the induced velocity of
    the whole network, with every free node excluded from the segments ending at its position (one stage of
    ``_network_convection`` for a network without rings)."""
    dev = nodes.device
    points = nodes[first:]
    velocity = _ambient(ambient, points, time).clone()
    if edges.shape[0] == 0 or points.shape[0] == 0:
        return velocity
    pairs = network.incident_pairs_device(nodes, edges, first)
    csr = network.exclusion_csr_device(points.shape[0], pairs)
    starts, directions, lengths = segments_of(nodes, edges)
    src = engine.Sources(starts, directions, lengths, gamma, radii, dev)
    tgt = engine.Targets(points, csr if csr[1].numel() else None, dev)
    if method == "direct":
        u, flags = engine.direct(src, tgt, model, singularity, precision, block, near)
    elif method == "tree":
        u, flags, _ = engine.tree_sum(src, tgt, model, singularity, precision, block, near, theta, order, leaf_size,
                                      3.0, "morton", far_counts=False)
    else:
        raise ValueError("method must be 'direct' or 'tree'")
    if bool(flags.any()):
        raise RuntimeError("a free node lies on a filament of the wake (the reference raises for this pair)")
    if not bool(torch.isfinite(u).all()):
        raise ValueError("velocity exceeds finite float64 range")
    return velocity.add_(u)


def convect(nodes, edges, gamma, radii, first, model, dt, ambient=(0.0, 0.0, 0.0), integrator="rk4", substeps=1,
            time=0.0, next_bound=None, **options):
    """Advance the free nodes nodes[first:] by dt (substeps explicit steps of the integrator) on the frozen graph;
    returns their new positions (device tensor [n - first, 3]).  The bound nodes nodes[:first] stay put, or move
    linearly to ``next_bound`` over the step (the reference's stage interpolation).  ``options`` go to
    ``network_velocity`` (method, precision, theta, order, ...)."""
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
    points = nodes[first:].clone()
    h = float(dt) / int(substeps)
    t0 = float(time)

    def rhs(current, t):
        stage_bound = bound if displacement is None or t == t0 else bound + ((t - t0) / float(dt)) * displacement
        return network_velocity(torch.cat((stage_bound, current)), edges, gamma, radii, first, model, ambient, t,
                                **options)

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
