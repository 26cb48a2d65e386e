"""Drop-in for the reference's GPU node quantities (vortex_cuda_moments, src/openfawe/aero/vortex_cuda_moments.py).

``device_node_quantities(order, lo, hi, starts, ends, alpha, length_vectors, radius, gamma)`` returns a dict of device
arrays ``centre, bound, core, m0, m1, m2, w1, t2, w2`` (float64; float32 copies rounded on the device with
``single=True``, the float64 ones then under ``m0_64`` ...) of ``vortex_tree.node_moments`` + ``node_contractions``
(vortex_tree.py:309-376, 425-447), computed by libbs_b200's ``bs_node_quantities``: chunked per-node reductions in a
fixed order, so repeated calls give the same bits; centre and core equal the CPU's bit for bit, the bounding radius
too (its squares are formed without contraction), the moments to rounding.  ``node_quantities`` copies them back.
The vortex vectors are gamma * length_vectors, which is how every caller forms ``alpha``; another ``alpha`` is refused.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import engine
from .devarray import DeviceArray

QUANTITIES = ("centre", "bound", "core", "m0", "m1", "m2", "w1", "t2", "w2")
_SHAPES = dict(centre=(3,), bound=(), core=(), m0=(3,), m1=(3, 3), m2=(3, 3, 3), w1=(3,), t2=(3,), w2=(3, 3))


class Statistics:
    """Counts for the tests: calls of ``device_node_quantities`` and library calls."""
    totals = dict(calls=0, launches=0)

    @classmethod
    def reset_totals(cls):
        cls.totals = dict(calls=0, launches=0)


def device_node_quantities(order, lo, hi, starts, ends, alpha, length_vectors, radius, gamma, *, single=False,
                           device_starts=None, device_order=None, device=None):
    dev = engine._device_of(device)
    lv = np.ascontiguousarray(length_vectors, dtype=np.float64).reshape(-1, 3)
    g = np.ascontiguousarray(gamma, dtype=np.float64).reshape(-1)
    if not np.array_equal(np.asarray(alpha, dtype=np.float64).reshape(-1, 3), g[:, None] * lv):
        raise ValueError("alpha must be gamma[:, None] * length_vectors")
    count, m = len(lo), len(g)
    Statistics.totals["calls"] += 1
    out = {k: torch.empty((count,) + _SHAPES[k], dtype=torch.float64, device=dev) for k in QUANTITIES}
    if count and m:
        d_order = (torch.as_tensor(device_order, device=dev).to(torch.int64).contiguous() if device_order is not None
                   else engine.i64(order, dev))
        d_starts = (torch.as_tensor(device_starts, device=dev).to(torch.float64).contiguous()
                    if device_starts is not None else engine.f64(starts, dev))
        # every device buffer stays referenced until the call has returned (a freed temporary's block can be handed
        # to the next allocation)
        args = [d_starts, engine.f64(ends, dev), engine.f64(lv, dev), engine.f64(g, dev), engine.f64(radius, dev)]
        d_lo, d_hi = engine.i64(lo, dev), engine.i64(hi, dev)
        L.check(L.library().bs_node_quantities(L.context(dev.index), m, *[engine._ptr(a) for a in args], count,
                                               engine._ptr(d_order), engine._ptr(d_lo), engine._ptr(d_hi),
                                               *[engine._ptr(out[k]) for k in QUANTITIES], engine._stream(dev)),
                "bs_node_quantities")
        Statistics.totals["launches"] += 1
    result = {k: DeviceArray(v) for k, v in out.items()}
    if single:
        for name in ("m0", "m1", "m2", "w1", "t2", "w2"):
            result[name + "_64"] = result[name]
            result[name] = DeviceArray(out[name].to(torch.float32))
    return result


def node_quantities(order, lo, hi, starts, ends, alpha, length_vectors, radius, gamma):
    """``device_node_quantities`` copied back to the host in float64: (centre, bound, core, m0, m1, m2, w1, t2, w2)."""
    d = device_node_quantities(order, lo, hi, starts, ends, alpha, length_vectors, radius, gamma)
    return tuple(d[name].copy_to_host() for name in QUANTITIES)
