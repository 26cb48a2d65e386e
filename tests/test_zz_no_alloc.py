"""The allocation-free direct sum (bs_direct_noalloc), called through the C ABI.

Some callers cannot allocate GPU memory while they run: a flight or control loop with a hard per-step deadline (an
allocation can stall in the driver, or fail once another framework's caching allocator holds the device), or a plugin
inside a host program that owns all device memory.  bs_direct_noalloc serves them with a fixed scratch array compiled
into the library.  Checked here:

* the config-1 lattice (FP64) against the reference's own numba output (tests/golden/direct_lattice.npz) within the
  reference's A1 bound, 1e-12 * sum_s |u_s| per target, and equal to the pooled bs_direct's result within the same bound;
* mixed and FP32 calls with exclusions against the pooled bs_direct within 1e-5 * sum_s |u_s| (the single-precision
  bound of the other parity tests), flags identical;
* a call at exactly the size limit (65,536 segments, mixed), where the last FP64 record ends where the FP32 records
  begin, against the pooled result;
* no device memory is taken by a call (free device memory and PyTorch's reserved bytes unchanged around it);
* sizes beyond the limit are rejected with BS_ERR_ARG.

This file is collected last on purpose; it must pass both alone in a fresh process and after the other tests, so it
sets up nothing it does not own.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scale(points, starts, directions, lengths, gamma, radius, model, csr=None, chunk=128):
    """sum_s |u_s| per target from the oracle's per-pair velocities (excluded pairs left out)."""
    out = np.zeros(len(points))
    for a in range(0, len(points), chunk):
        pairs, _ = O.pair_matrix(points[a:a + chunk], starts, directions, lengths, radius, model, False)
        mag = np.linalg.norm(pairs, axis=2) * np.abs(gamma)[None, :]
        if csr is not None:
            for p in range(a, min(a + chunk, len(points))):
                mag[p - a, csr[1][csr[0][p]:csr[0][p + 1]]] = 0.0
        out[a:a + chunk] = mag.sum(axis=1)
    return out


def _noalloc(lib, sources, targets, params, out, flags, stream):
    fn = lib.bs_direct_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 6
    return fn(ctypes.addressof(sources), ctypes.addressof(targets), ctypes.addressof(params),
              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(flags.data_ptr()), stream)


def _call(device, args, csr, precision):
    """One bs_direct_noalloc call on fresh NaN-filled outputs: (u, flags) as NumPy, the device memory the call took
    (free bytes lost, PyTorch bytes reserved), and the sources and targets it ran on."""
    import torch
    from openfawe_b200 import _lib, engine
    lib = _lib.library()
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    src = engine.Sources(*args[1:6], device)
    tgt = engine.Targets(args[0], csr, device)
    out = torch.full((tgt.n, 3), np.nan, dtype=torch.float64, device=device)
    flags = torch.full((tgt.n,), 7, dtype=torch.int8, device=device)
    params = engine.kernel_params(args[6], "raise", precision, 128, 3.0)
    s, t = src.struct(), tgt.struct()
    torch.cuda.synchronize(device)
    free0, reserved0 = torch.cuda.mem_get_info(device)[0], torch.cuda.memory_reserved(device)
    rc = _noalloc(lib, s, t, params, out, flags, stream)
    torch.cuda.synchronize(device)
    free1, reserved1 = torch.cuda.mem_get_info(device)[0], torch.cuda.memory_reserved(device)
    assert rc == 0, _lib.last_error()
    return out.cpu().numpy(), flags.cpu().numpy(), (free0 - free1, reserved1 - reserved0), src, tgt


def _pooled(device, src, tgt, model, precision):
    from openfawe_b200 import engine
    u, flags = engine.direct(src, tgt, model, "raise", precision)
    return u.cpu().numpy(), flags.cpu().numpy()


def _within(u, ref, scale, tol, what):
    err = np.linalg.norm(u - ref, axis=1)
    assert np.all(err <= tol * scale), (what, float(np.max(err / np.maximum(scale, 1e-300))))


def test_no_alloc_direct_on_calls_in_a_row(device):
    from openfawe_b200 import wakes
    lattice = wakes.lattice()
    lat_args = wakes.backend_args(lattice)
    g = golden("direct_lattice.npz")
    assert float(g["points_sum"]) == lattice["points"].sum() and float(g["starts_sum"]) == lattice["starts"].sum()
    lat_scale = _scale(*lat_args)
    e = golden("direct_exclusions.npz")
    ex_args = (e["points"], e["starts"], e["directions"], e["lengths"], e["gamma"], e["radius"], 2)
    ex_csr = (e["ptr"], e["seg"])
    ex_scale = _scale(*ex_args, csr=ex_csr)
    # the lattice twice (the second call sees the first call's records in the array), then smaller mixed and FP32
    # calls with exclusions (stale records beyond their segment count would show), each twice, then the lattice again
    seen = set()
    for step, (args, csr, precision, scale) in enumerate(((lat_args, None, "fp64", lat_scale),
                                                          (lat_args, None, "fp64", lat_scale),
                                                          (ex_args, ex_csr, "mixed", ex_scale),
                                                          (ex_args, ex_csr, "mixed", ex_scale),
                                                          (ex_args, ex_csr, "fp32", ex_scale),
                                                          (ex_args, ex_csr, "fp32", ex_scale),
                                                          (lat_args, None, "fp64", lat_scale))):
        u, flags, taken, src, tgt = _call(device, args, csr, precision)
        if precision in seen:  # a first call may load the library's device code; a repeated call takes nothing
            assert taken == (0, 0), (step, taken)
        seen.add(precision)
        ref, ref_flags = _pooled(device, src, tgt, args[6], precision)
        assert np.array_equal(flags, ref_flags), (step, precision)
        if precision == "fp64":
            assert not flags.any() and not bool(g["flag"])
            _within(u, g["u"], scale, 1e-12, "lattice vs the reference's numba direct sum")
            _within(u, ref, scale, 1e-12, "lattice vs bs_direct")
        else:
            _within(u, ref, scale, 1e-5, precision)


def test_no_alloc_at_the_size_limit(device):
    from openfawe_b200 import wakes
    case = wakes.rotor_sheet(300, seed=65536, targets=96)
    m = 65536
    assert len(case["starts"]) >= m
    args = (case["points"], *(case[k][:m] for k in ("starts", "directions", "lengths", "gamma", "radius")),
            case["model"])
    u, flags, taken, src, tgt = _call(device, args, None, "mixed")
    ref, ref_flags = _pooled(device, src, tgt, args[6], "mixed")
    assert np.array_equal(flags, ref_flags) and not flags.any()
    _within(u, ref, _scale(*args), 1e-5, "mixed at 65,536 segments")
    u2, _, taken2, _, _ = _call(device, args, None, "mixed")
    assert taken2 == (0, 0) and np.array_equal(u2, u)


def test_no_alloc_rejects_sizes_beyond_its_scratch(device):
    import torch
    from openfawe_b200 import _lib, engine
    lib = _lib.library()
    m = 65537
    rng = np.random.default_rng(1)
    d = rng.normal(size=(m, 3))
    sources = engine.Sources(rng.normal(size=(m, 3)), d / np.linalg.norm(d, axis=1)[:, None], np.ones(m),
                             np.ones(m), np.zeros(m), device)
    src = sources.struct()
    tgt = engine.Targets(np.zeros((4, 3)), None, device)
    out = torch.zeros((4, 3), dtype=torch.float64, device=device)
    flags = torch.zeros(4, dtype=torch.int8, device=device)
    params = engine.kernel_params(0, "raise", "fp64", 128, 3.0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    assert _noalloc(lib, src, tgt.struct(), params, out, flags, stream) == _lib.BS_ERR_ARG
    assert "65536" in _lib.last_error()
