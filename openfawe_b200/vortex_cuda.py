"""Drop-in for the reference's GPU direct-sum backend ``openfawe.aero.vortex_cuda`` (src/openfawe/aero/vortex_cuda.py).

Same public names and call signature: ``available``, ``probe_error``, ``Statistics``, ``cuda_sum(points, starts,
directions, lengths, gamma, radius, model, csr, singularity, settings, *, pairs_per_launch=None) -> (out, any_flag)``
(vortex_cuda.py:381-467), with the arrays validated by the caller (``segments_velocity``, vortex.py:421-465).  The
sum runs in the sm_100a kernel of libbs_b200 (``bs_direct``):

* ``fp64``: every pair in FP64, the reference's per-pair arithmetic (vortex_numba.pair_velocity);
* ``mixed``: FP32 pair arithmetic on two-float coordinates, FP64 re-evaluation of pairs within ``near`` core radii of a
  segment or near its axis (the reference's "suspect" pairs, vortex_cuda.py:23-24), FP64 per-target sums;
* ``fp32``: as ``mixed`` with FP32 per-target sums.

There is no CPU recomputation and no CPU fallback: where the reference sends suspect targets or whole calls to the CPU
(vortex_cuda.py:425-458) this backend evaluates the affected pairs in FP64 on the GPU.  Flags keep the reference's
meaning: the caller re-runs its NumPy reference to raise (vortex.py:488-492).  ``pairs_per_launch`` is accepted and
ignored (the reference splits launches for the Windows display watchdog; one launch covers the call here).
"""
import time

import numpy as np

FLAG_OK, FLAG_SINGULAR, FLAG_NONFINITE = 0, 1, 2
BLOCKS = (32, 64, 128, 256)
PRECISIONS = ("fp64", "mixed", "fp32")

_AVAILABLE = []
_PROBE_ERROR = []


def available():
    """True when a CUDA device can run this backend: torch sees a device and libbs_b200 initialises it (its probe
    kernel writes and reads back a value, as vortex_cuda.available does).  Cached."""
    if not _AVAILABLE:
        ok = False
        try:
            import torch
            if torch.cuda.is_available():
                from . import _lib
                _lib.context(torch.cuda.current_device())
                ok = True
            else:
                _PROBE_ERROR.append("torch.cuda.is_available() is False")
        except Exception as error:  # noqa: BLE001 - any driver, library or device problem means "not available"
            _PROBE_ERROR.append(f"{type(error).__name__}: {str(error)[:400]}")
        if not ok and not _PROBE_ERROR:
            _PROBE_ERROR.append("the device probe failed")
        _AVAILABLE.append(ok)
    return _AVAILABLE[0]


def probe_error():
    """Why ``available()`` said no (None when it said yes or was not asked)."""
    return _PROBE_ERROR[0] if _PROBE_ERROR else None


class Statistics:
    last = {}
    totals = dict(calls=0, suspect=0, suspect_max_per_call=0, cpu_fallback_calls=0, launches=0, fp64_pairs=0)

    @classmethod
    def reset_totals(cls):
        cls.totals = dict(calls=0, suspect=0, suspect_max_per_call=0, cpu_fallback_calls=0, launches=0, fp64_pairs=0)


def _check_settings(settings):
    precision = settings.precision
    if precision not in PRECISIONS:
        raise ValueError("cuda precision must be 'fp64', 'mixed' or 'fp32'")
    block = int(settings.block)
    if block not in BLOCKS:
        raise ValueError("cuda block must be 32, 64, 128 or 256")
    return precision, block, float(getattr(settings, "near", 3.0))


def to_host(device_tensor, shape, dtype):
    """An owned NumPy array holding a device tensor (one device-to-host copy)."""
    import torch
    host = np.empty(shape, dtype=dtype)
    if host.size:
        torch.from_numpy(host).copy_(device_tensor.reshape(shape))
    return host


def cuda_sum(points, starts, directions, lengths, gamma, radius, model, csr, singularity, settings, *,
             pairs_per_launch=None):
    """Return (velocity, any_flag) for validated inputs from segments_velocity (like direct_sum and tree_sum)."""
    if not available():
        raise ValueError(f"the cuda velocity backend needs a CUDA device ({probe_error()})")
    precision, block, near = _check_settings(settings)
    points = np.ascontiguousarray(points, dtype=np.float64)
    n, m = len(points), len(starts)
    if n == 0 or m == 0:
        Statistics.last = dict(points=n, segments=m, launches=0, suspect=0)
        return np.zeros((n, 3)), False
    import torch
    from . import engine
    device = torch.cuda.current_device()
    tick = time.perf_counter()
    sources = engine.Sources(starts, directions, lengths, gamma, radius, device)
    targets = engine.Targets(points, csr, device)
    upload_s = time.perf_counter() - tick
    tick = time.perf_counter()
    d_out, d_flags = engine.direct(sources, targets, int(model), singularity, precision, block, near)
    out = to_host(d_out, (n, 3), np.float64)
    flags = to_host(d_flags, (n,), np.int8)
    total_s = time.perf_counter() - tick
    stats = engine.last_stats(device)
    Statistics.last = dict(points=n, segments=m, launches=int(stats["launches"]), segments_per_launch=m, suspect=0,
                           fp64_pairs=int(stats["fp64_pairs"]), gpu_flagged_suspects=0,
                           longest_launch_s=stats["evaluate_ms"] * 1e-3, cpu_fallback=False, upload_s=upload_s,
                           evaluate_s=total_s, precision=precision)
    Statistics.totals["calls"] += 1
    Statistics.totals["launches"] += int(stats["launches"])
    Statistics.totals["fp64_pairs"] += int(stats["fp64_pairs"])
    return out, bool(np.any(flags))
