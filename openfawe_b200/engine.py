"""Device-resident interface of the B200 library: PyTorch CUDA tensors in, PyTorch CUDA tensors out.

The drop-in backends (``vortex_cuda.cuda_sum``, ``vortex_cuda_tree.cuda_tree_sum``) take NumPy arrays like the
reference's; this module is the layer below them, for callers that keep wakes in HBM across calls (build a tree once,
evaluate it at several target sets, or time the kernels without host copies).  All work is enqueued on the current
PyTorch stream of the tensors' device.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from .settings import PRECISION_CODES

_BLOCKS = (32, 64, 128, 256)


def _device_of(device):
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    if isinstance(device, int):
        return torch.device("cuda", device)
    return torch.device(device)


UPLOAD_MIN_BYTES = 1 << 20  # host arrays from this size up travel through bs_upload (threaded pinned staging)


def _upload(array, dtype, device):
    """Host NumPy array -> new device tensor through the library's pinned staging ring (bs_upload)."""
    out = torch.empty(array.shape, dtype=dtype, device=device)
    L.check(L.library().bs_upload(L.context(device.index), _ptr(out), array.ctypes.data_as(ctypes.c_void_p),
                                  array.nbytes, _stream(device)), "bs_upload")
    return out


def _to_device(a, np_dtype, dtype, device):
    if not isinstance(a, torch.Tensor):
        array = np.ascontiguousarray(a, dtype=np_dtype)
        if device.type == "cuda" and array.nbytes >= UPLOAD_MIN_BYTES:
            return _upload(array, dtype, device)
        a = torch.from_numpy(array if array.flags.writeable else array.copy())
    return a.to(device=device, dtype=dtype).contiguous()


def f64_many(arrays, device):
    """Several arrays as C-contiguous float64 tensors on `device`: the large host arrays go through one pass of the
    library's pinned staging ring (bs_upload_many), the rest as in f64."""
    device = _device_of(device)
    out = [None] * len(arrays)
    dst, src, nbytes, keep = [], [], [], []
    for i, a in enumerate(arrays):
        if device.type == "cuda" and not isinstance(a, torch.Tensor):
            array = np.ascontiguousarray(a, dtype=np.float64)
            if array.nbytes >= UPLOAD_MIN_BYTES:
                out[i] = torch.empty(array.shape, dtype=torch.float64, device=device)
                dst.append(out[i].data_ptr())
                src.append(array.ctypes.data)
                nbytes.append(array.nbytes)
                keep.append(array)
                continue
        out[i] = f64(a, device)
    if dst:
        k = len(dst)
        L.check(L.library().bs_upload_many(L.context(device.index), k, (ctypes.c_void_p * k)(*dst),
                                           (ctypes.c_void_p * k)(*src), (ctypes.c_size_t * k)(*nbytes),
                                           _stream(device)), "bs_upload_many")
    return out


def to_host_many(tensors, shapes, dtypes):
    """Owned NumPy arrays holding device tensors, copied through the library's pinned ring in one pass
    (bs_download_many); None entries give None."""
    out = [None if t is None else np.empty(shape, dtype=dtype) for t, shape, dtype in zip(tensors, shapes, dtypes)]
    pairs = [(h, t) for h, t in zip(out, tensors) if t is not None and h.size]
    if pairs:
        device = pairs[0][1].device
        k = len(pairs)
        views = [t.contiguous() for _, t in pairs]
        L.check(L.library().bs_download_many(L.context(device.index), k,
                                             (ctypes.c_void_p * k)(*[h.ctypes.data for h, _ in pairs]),
                                             (ctypes.c_void_p * k)(*[v.data_ptr() for v in views]),
                                             (ctypes.c_size_t * k)(*[h.nbytes for h, _ in pairs]), _stream(device)),
                "bs_download_many")
    return out


def f64(a, device):
    """A C-contiguous float64 tensor on `device` (copies only when needed)."""
    return _to_device(a, np.float64, torch.float64, _device_of(device))


def i64(a, device):
    return _to_device(a, np.int64, torch.int64, _device_of(device))


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() else ctypes.c_void_p(0)


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class Sources:
    """Directed segments resident on one device: starts [m,3], directions [m,3], lengths, gamma, radius [m]."""

    def __init__(self, starts, directions, lengths, gamma, radius, device=None):
        self.device = _device_of(device)
        starts, directions, lengths, gamma, radius = f64_many((starts, directions, lengths, gamma, radius), self.device)
        self.starts = starts.reshape(-1, 3)
        self.directions = directions.reshape(-1, 3)
        self.lengths = lengths.reshape(-1)
        self.gamma = gamma.reshape(-1)
        self.radius = radius.reshape(-1)
        self.m = int(self.starts.shape[0])

    def struct(self):
        return L.Sources(self.m, _ptr(self.starts), _ptr(self.directions), _ptr(self.lengths), _ptr(self.gamma),
                         _ptr(self.radius))


class Targets:
    """Target points [n,3] and optional exclusion CSR (ptr [n+1], seg [e], per-target sorted unique)."""

    def __init__(self, points, csr=None, device=None):
        self.device = _device_of(device)
        self.points = f64(points, self.device).reshape(-1, 3)
        self.n = int(self.points.shape[0])
        self.ex_ptr = self.ex_seg = None
        self.e = 0
        if csr is not None and len(csr[1]):
            self.ex_ptr = i64(csr[0], self.device)
            self.ex_seg = i64(csr[1], self.device)
            self.e = int(self.ex_seg.numel())

    def struct(self):
        return L.Targets(self.n, _ptr(self.points), _ptr(self.ex_ptr), _ptr(self.ex_seg), self.e)


def kernel_params(model, singularity="raise", precision="fp64", block=128, near=3.0):
    if int(block) not in _BLOCKS:
        raise ValueError("cuda block must be 32, 64, 128 or 256")
    code = PRECISION_CODES[precision] if isinstance(precision, str) else int(precision)
    return L.KernelParams(int(model), int(singularity == "raise"), code, int(block), float(near))


def tree_params(theta=0.5, order=2, leaf_size=32, clearance=3.0, kind="median", stack_limit=0):
    code = {"median": L.BS_TREE_MEDIAN, "morton": L.BS_TREE_MORTON}[kind] if isinstance(kind, str) else int(kind)
    return L.TreeParams(float(theta), int(order), int(leaf_size), float(clearance), code, int(stack_limit))


def direct(sources, targets, model, singularity="raise", precision="fp64", block=128, near=3.0):
    """Exact direct sum: returns (velocity [n,3] float64, flags [n] int8) device tensors."""
    dev = sources.device
    out = torch.empty((targets.n, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(targets.n, dtype=torch.int8, device=dev)
    src, tgt = sources.struct(), targets.struct()
    kp = kernel_params(model, singularity, precision, block, near)
    L.check(L.library().bs_direct(L.context(dev.index), ctypes.byref(src), ctypes.byref(tgt), ctypes.byref(kp),
                                  _ptr(out), _ptr(flags), _stream(dev)), "bs_direct")
    return out, flags


class Tree:
    """A tree on the device (freed with the object)."""

    def __init__(self, handle, sources, params):
        self._handle = handle
        self.sources = sources
        self.params = params
        self.count = int(L.library().bs_tree_count(handle))

    def __del__(self):
        handle, self._handle = getattr(self, "_handle", None), None
        if handle:
            try:
                L.library().bs_tree_free(handle)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass

    @property
    def handle(self):
        return self._handle

    def export(self):
        """The tree arrays in the reference's layout (vortex_tree.build_tree / node_moments / node_contractions) as
        NumPy arrays: order, lo, hi, left, right, centre, bound, core, m0, m1, m2, w1, t2, w2."""
        dev, c, m = self.sources.device, self.count, self.sources.m
        shapes = dict(order=(m,), lo=(c,), hi=(c,), left=(c,), right=(c,), centre=(c, 3), bound=(c,), core=(c,),
                      m0=(c, 3), m1=(c, 3, 3), m2=(c, 3, 3, 3), w1=(c, 3), t2=(c, 3), w2=(c, 3, 3))
        ints = ("order", "lo", "hi", "left", "right")
        t = {k: torch.empty(v, dtype=torch.int64 if k in ints else torch.float64, device=dev)
             for k, v in shapes.items()}
        L.check(L.library().bs_tree_export(self._handle, *[_ptr(t[k]) for k in shapes], _stream(dev)),
                "bs_tree_export")
        return {k: v.cpu().numpy() for k, v in t.items()}

    def keys(self):
        """Morton keys (input order, uint64) and their stable sort permutation (Morton trees only)."""
        dev, m = self.sources.device, self.sources.m
        keys = torch.empty(m, dtype=torch.int64, device=dev)
        order = torch.empty(m, dtype=torch.int64, device=dev)
        L.check(L.library().bs_tree_keys(self._handle, _ptr(keys), _ptr(order), _stream(dev)), "bs_tree_keys")
        return keys.cpu().numpy().view(np.uint64), order.cpu().numpy()


def build_tree(sources, theta=0.5, order=2, leaf_size=32, clearance=3.0, kind="median"):
    """Build a tree (median or Morton) with FP64 node moments on the device."""
    dev = sources.device
    params = tree_params(theta, order, leaf_size, clearance, kind)
    handle = ctypes.c_void_p()
    src = sources.struct()
    L.check(L.library().bs_tree_build(L.context(dev.index), ctypes.byref(src), ctypes.byref(params),
                                      ctypes.byref(handle), _stream(dev)), "bs_tree_build")
    return Tree(handle, sources, params)


def tree_from_arrays(sources, order, lo, hi, left, right):
    """A tree given as the reference's arrays (vortex_tree.build_tree output); moments computed on the device."""
    dev = sources.device
    arrays = [i64(a, dev) for a in (order, lo, hi, left, right)]
    handle = ctypes.c_void_p()
    src = sources.struct()
    L.check(L.library().bs_tree_from_arrays(L.context(dev.index), ctypes.byref(src), *[_ptr(a) for a in arrays],
                                            int(arrays[1].numel()), ctypes.byref(handle), _stream(dev)),
            "bs_tree_from_arrays")
    return Tree(handle, sources, tree_params())


def tree_eval(tree, targets, model, singularity="raise", precision="fp64", block=128, near=3.0, theta=0.5,
              order=2, clearance=3.0, stack_limit=0, far_counts=True):
    """Evaluate a tree at the targets: (velocity [n,3] float64, flags [n] int8, far counts [n] int64 or None)."""
    dev = tree.sources.device
    out = torch.empty((targets.n, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(targets.n, dtype=torch.int8, device=dev)
    far = torch.empty(targets.n, dtype=torch.int64, device=dev) if far_counts else None
    tp = tree_params(theta, order, tree.params.leaf_size, clearance, tree.params.kind, stack_limit)
    kp = kernel_params(model, singularity, precision, block, near)
    tgt = targets.struct()
    L.check(L.library().bs_tree_eval(L.context(dev.index), tree.handle, ctypes.byref(tp), ctypes.byref(tgt),
                                     ctypes.byref(kp), _ptr(out), _ptr(flags), _ptr(far), _stream(dev)),
            "bs_tree_eval")
    return out, flags, far


def tree_sum(sources, targets, model, singularity="raise", precision="mixed", block=128, near=3.0, theta=0.5,
             order=2, leaf_size=32, clearance=3.0, kind="median", stack_limit=0, far_counts=True):
    """Build, evaluate and free in one library call."""
    dev = sources.device
    out = torch.empty((targets.n, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(targets.n, dtype=torch.int8, device=dev)
    far = torch.empty(targets.n, dtype=torch.int64, device=dev) if far_counts else None
    tp = tree_params(theta, order, leaf_size, clearance, kind, stack_limit)
    kp = kernel_params(model, singularity, precision, block, near)
    src, tgt = sources.struct(), targets.struct()
    L.check(L.library().bs_tree_sum(L.context(dev.index), ctypes.byref(src), ctypes.byref(tp), ctypes.byref(tgt),
                                    ctypes.byref(kp), _ptr(out), _ptr(flags), _ptr(far), _stream(dev)),
            "bs_tree_sum")
    return out, flags, far


def tree_sum_host(points, starts, directions, lengths, gamma, radius, csr, model, singularity="raise",
                  precision="mixed", block=128, near=3.0, theta=0.5, order=2, leaf_size=32, clearance=3.0,
                  kind="median", stack_limit=0, device=None, far_counts=True):
    """tree_sum from and to host NumPy arrays in one library call (bs_tree_sum_host): returns (velocity [n,3] float64,
    flags [n] int8, far counts [n] int64 or None) as NumPy arrays.  csr = (ptr [n+1], seg [e]) or None."""
    dev = _device_of(device)
    c = lambda a, dt: np.ascontiguousarray(a, dtype=dt)  # noqa: E731
    points = c(points, np.float64).reshape(-1, 3)
    starts, directions = c(starts, np.float64).reshape(-1, 3), c(directions, np.float64).reshape(-1, 3)
    m = len(starts)
    lengths, gamma = c(lengths, np.float64).reshape(-1), c(gamma, np.float64).reshape(-1)
    radius = c(np.broadcast_to(np.asarray(radius, dtype=np.float64), (m,)), np.float64)
    n = len(points)
    ptr = seg = None
    if csr is not None and len(csr[1]):
        ptr, seg = c(csr[0], np.int64), c(csr[1], np.int64)
    out = np.empty((n, 3), dtype=np.float64)
    flags = np.empty(n, dtype=np.int8)
    far = np.empty(n, dtype=np.int64) if far_counts else None
    addr = lambda a: ctypes.c_void_p(a.ctypes.data if a is not None and a.size else 0)  # noqa: E731
    src = L.Sources(m, addr(starts), addr(directions), addr(lengths), addr(gamma), addr(radius))
    tgt = L.Targets(n, addr(points), addr(ptr), addr(seg), 0 if seg is None else len(seg))
    tp = tree_params(theta, order, leaf_size, clearance, kind, stack_limit)
    kp = kernel_params(model, singularity, precision, block, near)
    L.check(L.library().bs_tree_sum_host(L.context(dev.index), ctypes.byref(src), ctypes.byref(tp),
                                         ctypes.byref(tgt), ctypes.byref(kp), addr(out), addr(flags), addr(far),
                                         _stream(dev)), "bs_tree_sum_host")
    return out, flags, far


def last_stats(device=0):
    """Counters and device times of the last call on `device` (bs_last_stats)."""
    return L.stats(device)


# ---------------------------------------------------------------------------------------------------------------------
# Forests: many wakes in one tree (batched evaluation).
# ---------------------------------------------------------------------------------------------------------------------
def build_forest(sources, wake_ptr, leaf_size=32, order=2):
    """One Morton tree over concatenated wakes; wake w owns segments [wake_ptr[w], wake_ptr[w+1])."""
    dev = sources.device
    ptr = i64(wake_ptr, dev)
    params = tree_params(0.5, order, leaf_size, 3.0, "morton")
    handle = ctypes.c_void_p()
    src = sources.struct()
    L.check(L.library().bs_forest_build(L.context(dev.index), ctypes.byref(src), int(ptr.numel() - 1), _ptr(ptr),
                                        ctypes.byref(params), ctypes.byref(handle), _stream(dev)), "bs_forest_build")
    tree = Tree(handle, sources, params)
    tree.wake_ptr = ptr
    tree.nwakes = int(ptr.numel() - 1)
    return tree


def forest_roots(tree):
    roots = torch.empty(tree.nwakes, dtype=torch.int32, device=tree.sources.device)
    L.check(L.library().bs_forest_roots(tree.handle, _ptr(roots), _stream(tree.sources.device)), "bs_forest_roots")
    return roots.cpu().numpy()


def forest_eval(tree, targets, target_wake_ptr, model, singularity="raise", precision="mixed", block=128, near=3.0,
                theta=0.5, order=2, clearance=3.0, stack_limit=0, far_counts=True, exact=None):
    """Evaluate every wake of a forest at its own targets (targets of wake w: [target_wake_ptr[w], ...[w+1])).

    ``exact`` (bool per target, or None): targets summed exactly over their wake's segments (no far node accepted), in
    the same launch -- the batched form of the control-point induction (bs_forest_eval_exact)."""
    dev = tree.sources.device
    ptr = i64(target_wake_ptr, dev)
    out = torch.empty((targets.n, 3), dtype=torch.float64, device=dev)
    flags = torch.empty(targets.n, dtype=torch.int8, device=dev)
    far = torch.empty(targets.n, dtype=torch.int64, device=dev) if far_counts else None
    tp = tree_params(theta, order, tree.params.leaf_size, clearance, "morton", stack_limit)
    kp = kernel_params(model, singularity, precision, block, near)
    tgt = targets.struct()
    if exact is None:
        L.check(L.library().bs_forest_eval(L.context(dev.index), tree.handle, ctypes.byref(tp), ctypes.byref(tgt),
                                           _ptr(ptr), ctypes.byref(kp), _ptr(out), _ptr(flags), _ptr(far),
                                           _stream(dev)), "bs_forest_eval")
    else:
        mask = _exact_mask(exact, targets.n, dev)
        L.check(L.library().bs_forest_eval_exact(L.context(dev.index), tree.handle, ctypes.byref(tp),
                                                 ctypes.byref(tgt), _ptr(ptr), _ptr(mask), ctypes.byref(kp), _ptr(out),
                                                 _ptr(flags), _ptr(far), _stream(dev)), "bs_forest_eval_exact")
    return out, flags, far


def _exact_mask(exact, n, dev):
    mask = exact if isinstance(exact, torch.Tensor) else torch.as_tensor(np.asarray(exact, dtype=np.uint8))
    mask = mask.to(device=dev, dtype=torch.uint8).reshape(-1).contiguous()
    if mask.numel() != n:
        raise ValueError("exact mask: one entry per target")
    return mask


class Graph:
    """A captured forest (or tree) evaluation; ``launch()`` replays it on the current stream."""

    def __init__(self, tree, targets, target_wake_ptr, model, singularity="raise", precision="mixed", block=128,
                 near=3.0, theta=0.5, order=2, clearance=3.0, exact=None):
        dev = tree.sources.device
        self.tree, self.targets, self.device = tree, targets, dev
        self.ptr = None if target_wake_ptr is None else i64(target_wake_ptr, dev)
        self.exact = None if exact is None else _exact_mask(exact, targets.n, dev)
        self.out = torch.empty((targets.n, 3), dtype=torch.float64, device=dev)
        self.flags = torch.empty(targets.n, dtype=torch.int8, device=dev)
        self.far = torch.empty(targets.n, dtype=torch.int64, device=dev)
        tp = tree_params(theta, order, tree.params.leaf_size, clearance, "morton")
        kp = kernel_params(model, singularity, precision, block, near)
        tgt = targets.struct()
        handle = ctypes.c_void_p()
        torch.cuda.current_stream(dev).synchronize()
        if self.exact is None:
            L.check(L.library().bs_forest_graph(L.context(dev.index), tree.handle, ctypes.byref(tp), ctypes.byref(tgt),
                                                _ptr(self.ptr), ctypes.byref(kp), _ptr(self.out), _ptr(self.flags),
                                                _ptr(self.far), ctypes.byref(handle)), "bs_forest_graph")
        else:
            L.check(L.library().bs_forest_graph_exact(L.context(dev.index), tree.handle, ctypes.byref(tp),
                                                      ctypes.byref(tgt), _ptr(self.ptr), _ptr(self.exact),
                                                      ctypes.byref(kp), _ptr(self.out), _ptr(self.flags),
                                                      _ptr(self.far), ctypes.byref(handle)), "bs_forest_graph_exact")
        self._handle = handle

    def launch(self):
        L.check(L.library().bs_graph_launch(self._handle, _stream(self.device)), "bs_graph_launch")
        return self.out, self.flags, self.far

    def status(self):
        s = L.Stats()
        L.check(L.library().bs_graph_status(self._handle, ctypes.byref(s)), "bs_graph_status")
        return s.as_dict()

    def __del__(self):
        handle, self._handle = getattr(self, "_handle", None), None
        if handle:
            try:
                L.library().bs_graph_free(handle)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
