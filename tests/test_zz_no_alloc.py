"""The allocation-free direct sum (bs_direct_noalloc) against the pooled one (bs_direct), through the C ABI.

bs_direct_noalloc serves callers that must not allocate GPU memory while they run (a control loop with a hard step
deadline, or a plugin in a host that owns the device's memory): its scratch is a fixed array inside the library.
This file is collected last on purpose; it must pass both alone in a fresh process and after the other tests, so it
sets up nothing it does not own.  Tolerance: the FP64 bound of the other parity tests, 1e-12 * sum_s |u_s| per target;
1e-5 * sum_s |u_s| for the mixed precision.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _scale(points, starts, directions, lengths, gamma, radius, model):
    pairs, _ = O.pair_matrix(points, starts, directions, lengths, radius, model, False)
    return (np.linalg.norm(pairs, axis=2) * np.abs(gamma)[None, :]).sum(axis=1)


def _noalloc(lib, sources, targets, params, out, flags, stream):
    fn = lib.bs_direct_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 6
    return fn(ctypes.addressof(sources), ctypes.addressof(targets), ctypes.addressof(params),
              ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(flags.data_ptr()), stream)


def test_no_alloc_direct_matches_pooled_direct_on_two_calls(device):
    import torch
    from openfawe_b200 import _lib, engine, wakes
    lib = _lib.library()
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    # two different calls in a row: a bigger FP64 one, then a smaller mixed one (stale records would show)
    g = golden("direct_exclusions.npz")
    lattice = wakes.lattice()
    cases = [(wakes.backend_args(lattice), None, "fp64", 1e-12),
             ((g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2),
              (g["ptr"], g["seg"]), "mixed", 1e-5)]
    for args, csr, precision, tol in cases:
        points, model = args[0], args[6]
        src = engine.Sources(*args[1:6], device)
        tgt = engine.Targets(points, csr, device)
        out = torch.full((tgt.n, 3), np.nan, dtype=torch.float64, device=device)
        flags = torch.full((tgt.n,), 7, dtype=torch.int8, device=device)
        params = engine.kernel_params(model, "raise", precision, 128, 3.0)
        rc = _noalloc(lib, src.struct(), tgt.struct(), params, out, flags, stream)
        assert rc == 0, _lib.last_error()
        ref, ref_flags = engine.direct(src, tgt, model, "raise", precision)
        u, r = out.cpu().numpy(), ref.cpu().numpy()
        assert np.array_equal(flags.cpu().numpy(), ref_flags.cpu().numpy())
        scale = _scale(*args)
        if csr is not None:
            for p in range(len(points)):
                excluded = csr[1][csr[0][p]:csr[0][p + 1]]
                pairs, _ = O.pair_matrix(points[p:p + 1], *args[1:4], args[5], model, False)
                scale[p] -= (np.linalg.norm(pairs[0, excluded], axis=1) * np.abs(args[4][excluded])).sum()
        assert np.all(np.linalg.norm(u - r, axis=1) <= tol * scale), precision


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
