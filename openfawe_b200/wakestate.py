"""Frozen wake states: the ``state_<step>.npz`` format the reference's benchmark reads
(paper1/scripts/convergence/local_benchmark.py:56-62) -- nodes [N,3], edges [E,2], gamma [E], radii [E] (or one
value), first (the bound-node count; the free nodes nodes[first:] are the targets), speed (the reference speed the
benchmark divides errors by), core_model, exclusions [e,2] (point, segment) -- loaded onto the device and evaluated
as the benchmark's ``segments_velocity(points, nodes, edges, gamma, model=core_model, core_radius=radii,
exclusions=exclusions)``.

Segments are formed on the host exactly as ``segments_velocity`` forms them (vortex.py:460-465), so the device
arrays equal the reference's inputs bit for bit; the exclusion CSR is built on the device (``bs_exclusion_csr``).
"""
import numpy as np
import torch

from . import engine, network

KEYS = ("nodes", "edges", "gamma", "radii", "first", "speed", "core_model", "exclusions")


def save_state(path, nodes, edges, gamma, radii, first, speed, core_model, exclusions=None):
    """Write a frozen wake state in the benchmark's format (compressed npz)."""
    exclusions = np.zeros((0, 2), dtype=np.int64) if exclusions is None else np.asarray(exclusions, dtype=np.int64)
    np.savez_compressed(path, nodes=np.asarray(nodes, dtype=np.float64), edges=np.asarray(edges, dtype=np.int64),
                        gamma=np.asarray(gamma, dtype=np.float64), radii=np.asarray(radii, dtype=np.float64),
                        first=np.int64(first), speed=np.float64(speed), core_model=np.int64(core_model),
                        exclusions=exclusions.reshape(-1, 2))


def load_state(path):
    """The state's arrays as a dict (NumPy), checked for the shapes the benchmark relies on."""
    with np.load(path) as data:
        missing = [k for k in KEYS if k not in data.files]
        if missing:
            raise ValueError(f"wake state {path}: missing {', '.join(missing)}")
        state = {k: data[k] for k in KEYS}
    nodes, edges = np.asarray(state["nodes"], dtype=np.float64), np.asarray(state["edges"], dtype=np.int64)
    if nodes.ndim != 2 or nodes.shape[1] != 3 or edges.ndim != 2 or edges.shape[1] != 2:
        raise ValueError("wake state: nodes must be [N,3] and edges [E,2]")
    first = int(state["first"])
    if not 0 <= first <= len(nodes) or (edges.size and (edges.min() < 0 or edges.max() >= len(nodes))):
        raise ValueError("wake state: first or an edge index out of range")
    state.update(nodes=nodes, edges=edges, first=first, speed=float(state["speed"]),
                 core_model=int(state["core_model"]),
                 exclusions=np.asarray(state["exclusions"], dtype=np.int64).reshape(-1, 2))
    return state


class FrozenWake:
    """A loaded state resident on one device: segments, target points and the exclusion CSR."""

    def __init__(self, state, device=None):
        if isinstance(state, str):
            state = load_state(state)
        self.state = state
        self.device = engine._device_of(device)
        nodes, edges = state["nodes"], state["edges"]
        starts = nodes[edges[:, 0]]
        delta = nodes[edges[:, 1]] - starts
        lengths = np.hypot(np.hypot(delta[..., 0], delta[..., 1]), delta[..., 2])
        if np.any(lengths == 0):
            raise ValueError("zero-length segment")
        directions = delta / lengths[:, None]
        radii = np.broadcast_to(np.asarray(state["radii"], dtype=np.float64), (len(edges),))
        self.model = int(state["core_model"])
        self.first = int(state["first"])
        self.sources = engine.Sources(starts, directions, lengths, state["gamma"], np.ascontiguousarray(radii),
                                      self.device)
        points = nodes[self.first:]
        pairs = state["exclusions"]
        if len(pairs) and (pairs[:, 0].max() >= len(points) or pairs[:, 1].max() >= len(edges) or pairs.min() < 0):
            raise ValueError("exclusion index out of range")
        csr = None
        if len(pairs):
            csr = network.exclusion_csr_device(len(points), engine.i64(pairs, self.device).reshape(-1, 2))
        self.targets = engine.Targets(points, csr, self.device)

    @property
    def speed(self):
        return float(self.state["speed"])

    def velocity(self, method="tree", precision="mixed", singularity="raise", theta=0.1, order=3, leaf_size=32,
                 block=128, near=3.0):
        """Induced velocity at the free nodes (device tensor [n, 3]) and the per-point flags."""
        if method == "direct":
            return engine.direct(self.sources, self.targets, self.model, singularity, precision, block, near)
        if method != "tree":
            raise ValueError("method must be 'direct' or 'tree'")
        u, flags, _ = engine.tree_sum(self.sources, self.targets, self.model, singularity, precision, block, near,
                                      theta, order, leaf_size, 3.0, "morton", far_counts=False)
        return u, flags

    def error_over_speed(self, u, reference):
        """max |u - reference| / speed, the benchmark's error measure."""
        u = u.cpu().numpy() if isinstance(u, torch.Tensor) else np.asarray(u)
        return float(np.max(np.abs(u - np.asarray(reference))) / self.speed)
