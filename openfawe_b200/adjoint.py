"""Differentiation of the induced velocity: hand-written adjoints behind torch.autograd.

``InducedVelocity.apply(points, starts, ends, gamma, radius, ...)`` returns the induced velocity [n,3] of directed
segments A->B; its backward returns d(w . u) with respect to the targets, both endpoints and the circulations for the
incoming cotangent w, recomputing every pair term rather than storing it:

* forward ``method='direct'`` (the exact sum): ``bs_adjoint_direct``, FP64;
* forward ``method='tree'``: ``bs_tree_adjoint``, the derivative of the tree sum the forward evaluated -- the same
  tree, accepted nodes and near pairs, with the far field differentiated through the node moments down to the segments
  (node centres and acceptance decisions held fixed).

Every core model (0..5) in both adjoints; the tree adjoint takes the models the reference's tree code does not accept
(Vatistas, offset, Rosenhead-Moore) with FP64 near pairs.  The reference has no adjoint.
"""
import ctypes

import torch

from . import _lib as L
from . import engine

_SIGNATURE = (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64] + [ctypes.c_void_p] * 6
              + [ctypes.c_int64, ctypes.c_int] + [ctypes.c_void_p] * 6)


def _fn():
    lib = L.library()
    fn = lib.bs_adjoint_direct
    fn.restype, fn.argtypes = _SIGNATURE
    return fn


def segments_from_endpoints(starts, ends):
    """(starts, unit directions, lengths) of A->B segments, formed as the reference forms them (vortex.py:460-465)."""
    delta = ends - starts
    lengths = torch.hypot(torch.hypot(delta[:, 0], delta[:, 1]), delta[:, 2])
    return starts, delta / lengths[:, None], lengths


def adjoint_direct(points, starts, ends, gamma, radius, model, cotangent, csr=None, need=(True, True, True, True)):
    """(grad_points, grad_starts, grad_ends, grad_gamma) of sum_p cotangent_p . u_p; float64 device tensors."""
    dev = points.device
    p = engine.f64(points, dev).reshape(-1, 3)
    a = engine.f64(starts, dev).reshape(-1, 3)
    b = engine.f64(ends, dev).reshape(-1, 3)
    g = engine.f64(gamma, dev).reshape(-1)
    r = engine.f64(radius, dev).reshape(-1)
    w = engine.f64(cotangent, dev).reshape(-1, 3)
    n, m = p.shape[0], a.shape[0]
    outs = [torch.empty((n, 3), dtype=torch.float64, device=dev) if need[0] else None,
            torch.empty((m, 3), dtype=torch.float64, device=dev) if need[1] else None,
            torch.empty((m, 3), dtype=torch.float64, device=dev) if need[2] else None,
            torch.empty(m, dtype=torch.float64, device=dev) if need[3] else None]
    ex_ptr = ex_seg = None
    e = 0
    if csr is not None and len(csr[1]):
        ex_ptr, ex_seg = engine.i64(csr[0], dev), engine.i64(csr[1], dev)
        e = int(ex_seg.numel())
    P = engine._ptr
    L.check(_fn()(L.context(dev.index), n, P(p), m, P(a), P(b), P(g), P(r), P(ex_ptr), P(ex_seg), e, int(model), P(w),
                  *[P(t) for t in outs], engine._stream(dev)), "bs_adjoint_direct")
    return tuple(outs)


def adjoint_tree(points, starts, ends, gamma, radius, model, cotangent, csr=None, precision="mixed", theta=0.215,
                 order=5, leaf_size=384, clearance=3.0, kind="morton", block=128, near=3.0,
                 need=(True, True, True, True)):
    """(grad_points, grad_starts, grad_ends, grad_gamma) of sum_p cotangent_p . u_p for u the tree sum with these
    settings (``engine.tree_sum``); float64 device tensors.  ``precision`` selects the near pairs' arithmetic ('mixed':
    FP32 with FP64 where the forward takes FP64; 'fp64': all FP64); the far field's derivatives are FP64."""
    dev = points.device if isinstance(points, torch.Tensor) else engine._device_of(None)
    a = engine.f64(starts, dev).reshape(-1, 3)
    b = engine.f64(ends, dev).reshape(-1, 3)
    s, d, length = segments_from_endpoints(a, b)
    src = engine.Sources(s, d, length, engine.f64(gamma, dev).reshape(-1), engine.f64(radius, dev).reshape(-1), dev)
    tgt = engine.Targets(points, csr, dev)
    w = engine.f64(cotangent, dev).reshape(-1, 3)
    n, m = tgt.n, src.m
    outs = [torch.empty((n, 3), dtype=torch.float64, device=dev) if need[0] else None,
            torch.empty((m, 3), dtype=torch.float64, device=dev) if need[1] else None,
            torch.empty((m, 3), dtype=torch.float64, device=dev) if need[2] else None,
            torch.empty(m, dtype=torch.float64, device=dev) if need[3] else None]
    tp = engine.tree_params(theta, order, leaf_size, clearance, kind)
    kp = engine.kernel_params(model, "raise", precision, block, near)
    srcs, tgts = src.struct(), tgt.struct()
    P = engine._ptr
    L.check(L.library().bs_tree_adjoint(L.context(dev.index), ctypes.byref(srcs), ctypes.byref(tp),
                                        ctypes.byref(tgts), ctypes.byref(kp), P(w), *[P(t) for t in outs],
                                        engine._stream(dev)), "bs_tree_adjoint")
    return tuple(outs)


class InducedVelocity(torch.autograd.Function):
    """u = induced velocity of segments (starts -> ends) with circulations gamma at the points.

    Arguments after the tensors: model, singularity, method ('direct' or 'tree'), precision, tree options (theta,
    order, leaf_size, clearance, kind) and the exclusion CSR (or None)."""

    @staticmethod
    def forward(ctx, points, starts, ends, gamma, radius, model=2, singularity="raise", method="tree",
                precision="mixed", theta=0.04, order=2, leaf_size=32, clearance=3.0, kind="morton", csr=None):
        dev = points.device
        s, d, length = segments_from_endpoints(starts.detach().to(torch.float64), ends.detach().to(torch.float64))
        src = engine.Sources(s, d, length, gamma.detach(), radius.detach(), dev)
        tgt = engine.Targets(points.detach(), csr, dev)
        if method == "direct":
            u, _ = engine.direct(src, tgt, model, singularity, precision)
        else:
            u, _, _ = engine.tree_sum(src, tgt, model, singularity, precision, theta=theta, order=order,
                                      leaf_size=leaf_size, clearance=clearance, kind=kind, far_counts=False)
        ctx.save_for_backward(points, starts, ends, gamma, radius)
        ctx.model, ctx.csr = model, csr
        ctx.tree = None if method == "direct" else dict(precision=precision, theta=theta, order=order,
                                                         leaf_size=leaf_size, clearance=clearance, kind=kind)
        return u.to(points.dtype)

    @staticmethod
    def backward(ctx, grad_u):
        points, starts, ends, gamma, radius = ctx.saved_tensors
        need = tuple(bool(v) for v in ctx.needs_input_grad[:4])
        args = (points.detach(), starts.detach(), ends.detach(), gamma.detach(), radius.detach(), ctx.model,
                grad_u.detach(), ctx.csr)
        if ctx.tree is None:
            gx, ga, gb, gg = adjoint_direct(*args, need=need)
        else:
            gx, ga, gb, gg = adjoint_tree(*args, need=need, **ctx.tree)
        cast = lambda t, like: None if t is None else t.to(like.dtype)  # noqa: E731
        return (cast(gx, points), cast(ga, starts), cast(gb, ends), cast(gg, gamma), None, None, None, None, None,
                None, None, None, None, None, None)


def induced_velocity(points, starts, ends, gamma, radius, **options):
    """Differentiable induced velocity (see InducedVelocity)."""
    return InducedVelocity.apply(points, starts, ends, gamma, radius, *[options.get(k, v) for k, v in (
        ("model", 2), ("singularity", "raise"), ("method", "tree"), ("precision", "mixed"), ("theta", 0.04),
        ("order", 2), ("leaf_size", 32), ("clearance", 3.0), ("kind", "morton"), ("csr", None))])
