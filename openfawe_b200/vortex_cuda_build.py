"""Drop-in for the reference's GPU tree build (vortex_cuda_build, src/openfawe/aero/vortex_cuda_build.py).

``device_build_tree(mid, leaf_size)`` returns ``(device order, order, lo, hi, left, right, node_count)`` whose host
arrays equal ``vortex_tree.build_tree(mid, leaf_size)``'s element for element (vortex_tree.py:208-241: median split
along the longest midpoint-box axis, lower axis on ties, stable order, depth-first numbering).  The splitting runs on
the device through libbs_b200's ``bs_median_topology`` (radix sorts of dense coordinate ranks per level).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import engine
from .devarray import DeviceArray


class Statistics:
    """Counts for the tests: calls of ``device_build_tree`` and library calls."""
    totals = dict(calls=0, launches=0, levels=0)

    @classmethod
    def reset_totals(cls):
        cls.totals = dict(calls=0, launches=0, levels=0)


def device_build_tree(mid, leaf_size, *, device_mid=None, device=None):
    mid = np.ascontiguousarray(mid, dtype=np.float64).reshape(-1, 3)
    leaf_size = int(leaf_size)
    if leaf_size < 1:
        raise ValueError("leaf_size must be positive")
    n = mid.shape[0]
    dev = engine._device_of(device)
    if device_mid is not None:
        d_mid = torch.as_tensor(device_mid, device=dev).to(torch.float64).reshape(-1, 3).contiguous()
    else:
        d_mid = engine.f64(mid, dev).reshape(-1, 3)
    Statistics.totals["calls"] += 1
    capacity = 4 * (n // leaf_size + 1) + 1
    order = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    arrays = [torch.empty(capacity, dtype=torch.int64, device=dev) for _ in range(4)]
    count = ctypes.c_int64(0)
    L.check(L.library().bs_median_topology(L.context(dev.index), n, engine._ptr(d_mid), leaf_size, engine._ptr(order),
                                           *[engine._ptr(a) for a in arrays], capacity, ctypes.byref(count),
                                           engine._stream(dev)), "bs_median_topology")
    Statistics.totals["launches"] += 1
    c = count.value
    if c > capacity:
        raise RuntimeError(f"bs_median_topology: {c} nodes exceed the capacity {capacity}")
    lo, hi, left, right = (a[:c].cpu().numpy() for a in arrays)
    order = order[:n]
    return DeviceArray(order), order.cpu().numpy(), lo, hi, left, right, c
