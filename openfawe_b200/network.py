"""Exclusion bookkeeping of the wake network on the GPU (libbs_b200 ``bs_incident_pairs`` / ``bs_exclusion_csr``).

Drop-ins for the reference's compiled bookkeeping that feeds every large sum of a free-wake step:

* ``incident_pairs(nodes, edges, first)`` -- network_numba.incident_pairs (src/openfawe/aero/network_numba.py:242-256):
  the (free point, segment) pairs whose point coincides bit for bit with an end of the segment, in the reference's
  order (segment, end, then increasing point).
* ``exclusion_csr(point_count, pairs)`` -- vortex_numba.exclusion_csr (src/openfawe/aero/vortex_numba.py:228-243): the
  per-point sorted unique excluded segments as ``(pointer, segments)``.

Both take and return NumPy arrays like the reference's; ``*_device`` variants take and return device tensors so that a
step can keep its exclusions resident and hand them straight to ``engine.Targets``.
"""
import ctypes
import operator

import numpy as np
import torch

from . import _lib as L
from . import engine


def _device(device):
    return engine._device_of(device)


def incident_pairs_device(nodes, edges, first, capacity=None):
    """nodes [n,3] float64 and edges [e,2] int64 device tensors -> pairs [k,2] int64 device tensor."""
    dev = nodes.device
    n, e = int(nodes.shape[0]), int(edges.shape[0])
    if not 0 <= int(first) <= n:
        raise ValueError("first must lie in [0, len(nodes)]")
    capacity = 2 * e + 16 if capacity is None else int(capacity)
    count = ctypes.c_int64(0)
    fn = L.library().bs_incident_pairs
    ctx = L.context(dev.index)
    for _ in range(2):
        pairs = torch.empty((max(capacity, 1), 2), dtype=torch.int64, device=dev)
        L.check(fn(ctx, engine._ptr(nodes), n, engine._ptr(edges), e, int(first), engine._ptr(pairs), capacity,
                   ctypes.byref(count), engine._stream(dev)), "bs_incident_pairs")
        if count.value <= capacity:
            return pairs[:count.value]
        capacity = count.value
    raise RuntimeError("bs_incident_pairs: pair count changed between calls")


def incident_pairs(nodes, edges, first, device=None):
    """Exclusion pairs of wake._network_convection as an (e, 2) int64 NumPy array (network_numba.incident_pairs)."""
    nodes = np.asarray(nodes, dtype=np.float64)
    edges = np.asarray(edges, dtype=np.int64)
    if nodes.ndim != 2 or nodes.shape[1] != 3 or edges.ndim != 2 or edges.shape[1] != 2:
        raise ValueError("incident_pairs needs (n, 3) nodes and (e, 2) edges")
    dev = _device(device)
    pairs = incident_pairs_device(engine.f64(nodes, dev).reshape(-1, 3), engine.i64(edges, dev).reshape(-1, 2),
                                  int(first))
    return np.ascontiguousarray(pairs.cpu().numpy())


def exclusion_csr_device(point_count, pairs):
    """pairs [e,2] int64 device tensor -> (ptr [point_count+1], seg [unique]) int64 device tensors."""
    dev = pairs.device
    e = int(pairs.shape[0])
    ptr = torch.empty(point_count + 1, dtype=torch.int64, device=dev)
    seg = torch.empty(max(e, 1), dtype=torch.int64, device=dev)
    count = ctypes.c_int64(0)
    L.check(L.library().bs_exclusion_csr(L.context(dev.index), int(point_count), engine._ptr(pairs), e,
                                         engine._ptr(ptr), engine._ptr(seg), ctypes.byref(count),
                                         engine._stream(dev)), "bs_exclusion_csr")
    return ptr, seg[:count.value]


def exclusion_csr(point_count, pairs, device=None):
    """Per-point sorted unique excluded segment ids from an (e, 2) (point, segment) array (vortex_numba.exclusion_csr).

    A point outside [0, point_count) raises ValueError, as the reference's fallback does."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        return np.zeros(point_count + 1, dtype=np.int64), np.zeros(0, dtype=np.int64)
    count = operator.index(point_count)
    dev = _device(device)
    ptr, seg = exclusion_csr_device(count, engine.i64(pairs, dev).reshape(-1, 2))
    return ptr.cpu().numpy(), np.ascontiguousarray(seg.cpu().numpy())
