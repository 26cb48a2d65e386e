"""Unit-circulation influence operators on the GPU (libbs_b200 ``bs_pair_matrix``, ``bs_assemble_columns``,
``bs_ring_columns``).

``pair_matrix`` and ``assemble_columns`` keep the reference's signatures (vortex_numba.pair_matrix / assemble_columns,
src/openfawe/aero/vortex_numba.py:271-308: NumPy outputs filled in place), so vsm_wake's batched ring and cross-class
operators (src/openfawe/aero/vsm_wake.py:123-252) can call them unchanged; ``ring_columns`` does both in one pass
without storing the [n, m, 3] pair matrix.  Pair values are the FP64 pair of the direct sum (within 1e-12 of the
reference's per pair); column sums run in the reference's order, so equal pairs give equal columns bit for bit.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import engine


def _sources(starts, directions, lengths, radius, dev):
    m = len(lengths)
    return engine.Sources(starts, directions, lengths, np.zeros(m) if not isinstance(lengths, torch.Tensor)
                          else torch.zeros(m, dtype=torch.float64, device=dev), radius, dev)


def _columns(column_ptr, column_segment, column_sign, m):
    ptr = np.asarray(column_ptr, dtype=np.int64)
    seg = np.asarray(column_segment, dtype=np.int64)
    sign = np.asarray(column_sign, dtype=np.float64)
    if ptr.ndim != 1 or len(ptr) < 1 or seg.ndim != 1 or sign.shape != seg.shape:
        raise ValueError("column layout: pointer [columns+1], segment and sign [entries] arrays")
    if np.any(np.diff(ptr) < 0) or ptr[0] < 0 or ptr[-1] > len(seg):
        raise ValueError("column pointer must be non-decreasing within [0, entries]")
    if len(seg) and (seg.min() < 0 or seg.max() >= m):
        raise ValueError("column segment outside [0, segment count)")
    return ptr, seg, sign


def pair_matrix_device(points, sources, model, raise_singular=True):
    """(pairs [n, m, 3], flags [n]) device tensors for `sources` (an ``engine.Sources``; its gamma is not read)."""
    dev = sources.device
    pts = engine.f64(points, dev).reshape(-1, 3)
    n, m = int(pts.shape[0]), sources.m
    out = torch.empty((n, m, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(n, dtype=torch.int8, device=dev)
    src = sources.struct()
    L.check(L.library().bs_pair_matrix(L.context(dev.index), n, engine._ptr(pts), ctypes.byref(src), int(model),
                                       int(bool(raise_singular)), engine._ptr(out), engine._ptr(flags),
                                       engine._stream(dev)), "bs_pair_matrix")
    return out, flags


def pair_matrix(points, starts, directions, lengths, radius, model, raise_singular, out, flags, device=None):
    """out[p, s, :] = unit-circulation velocity of segment s at point p; flags per point (vortex_numba.pair_matrix)."""
    dev = engine._device_of(device)
    pairs, f = pair_matrix_device(points, _sources(starts, directions, lengths, radius, dev), model, raise_singular)
    out[...] = pairs.cpu().numpy()
    flags[...] = f.cpu().numpy()


def assemble_columns(pairs, column_ptr, column_segment, column_sign, out, device=None):
    """out[p, j, :] = sum_k sign_k * pairs[p, segment_k, :], sequential in k from 0.0 (vortex_numba.assemble_columns)."""
    dev = engine._device_of(device)
    pairs_t = engine.f64(pairs, dev)
    n, m = int(pairs_t.shape[0]), int(pairs_t.shape[1])
    ptr, seg, sign = _columns(column_ptr, column_segment, column_sign, m)
    columns = len(ptr) - 1
    res = torch.empty((n, columns, 3), dtype=torch.float64, device=dev)
    ptr_t, seg_t, sign_t = engine.i64(ptr, dev), engine.i64(seg, dev), engine.f64(sign, dev)
    L.check(L.library().bs_assemble_columns(L.context(dev.index), n, m, engine._ptr(pairs_t), columns,
                                            engine._ptr(ptr_t), engine._ptr(seg_t), engine._ptr(sign_t),
                                            engine._ptr(res), engine._stream(dev)), "bs_assemble_columns")
    out[...] = res.cpu().numpy()


def ring_columns(points, starts, directions, lengths, radius, model, raise_singular, column_ptr, column_segment,
                 column_sign, device=None):
    """(columns [n, J, 3], flags [n]) NumPy arrays: pair_matrix + assemble_columns in one pass."""
    dev = engine._device_of(device)
    src = _sources(starts, directions, lengths, radius, dev)
    ptr, seg, sign = _columns(column_ptr, column_segment, column_sign, src.m)
    pts = engine.f64(points, dev).reshape(-1, 3)
    n, columns = int(pts.shape[0]), len(ptr) - 1
    res = torch.empty((n, columns, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(n, dtype=torch.int8, device=dev)
    ptr_t, seg_t, sign_t = engine.i64(ptr, dev), engine.i64(seg, dev), engine.f64(sign, dev)
    s = src.struct()
    L.check(L.library().bs_ring_columns(L.context(dev.index), n, engine._ptr(pts), ctypes.byref(s), int(model),
                                        int(bool(raise_singular)), columns, engine._ptr(ptr_t), engine._ptr(seg_t),
                                        engine._ptr(sign_t), engine._ptr(res), engine._ptr(flags),
                                        engine._stream(dev)), "bs_ring_columns")
    return res.cpu().numpy(), flags.cpu().numpy()
