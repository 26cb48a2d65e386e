"""CPU oracle of the Biot-Savart hot path -- TEST INFRASTRUCTURE ONLY.

NumPy/ctypes front end of ``oracle/liboracle.so`` (``bs_oracle.c``: the reference's FP64 algorithms restated in C,
``morton_oracle.c``: the CPU recomputation of the B200 build's Morton tree).  Only the tests, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` import this module, as the checker; the product package never does.

Functions mirror the reference's backend functions (paths inside the reference project):
``direct_sum`` (src/openfawe/aero/vortex_numba.py:246-260), ``exclusion_csr`` (:228-243), ``pair_matrix`` (:271-287),
``build_tree`` (src/openfawe/aero/vortex_tree.py:208-241), ``node_moments`` (:309-376), ``node_contractions``
(:425-447), ``far_velocity`` (:450-497), ``tree_velocity`` (:508-568) and ``tree_sum`` (:588-626).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "liboracle.so")
SUPPORTED_TREE_MODELS = (0, 1, 2)
_LIB = []

_d = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_i8 = ctypes.POINTER(ctypes.c_int8)
_I = ctypes.c_int64


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    if not _LIB:
        if not os.path.exists(LIBRARY):
            build()
        handle = ctypes.CDLL(LIBRARY)
        sig = {
            "orc_pairs": (None, [_I, _d, _d, _d, _d, _d, _d, ctypes.c_int, ctypes.c_int, _d, _i8]),
            "orc_direct_sum": (None, [_I, _d, _I, _d, _d, _d, _d, _d, ctypes.c_int, ctypes.c_int, _i64, _i64, _d, _i8,
                                      ctypes.c_int]),
            "orc_pair_matrix": (None, [_I, _d, _I, _d, _d, _d, _d, ctypes.c_int, ctypes.c_int, _d, _i8]),
            "orc_exclusion_csr": (_I, [_I, _I, _i64, _i64, _i64]),
            "orc_incident_pairs": (_I, [_I, _d, _I, _i64, _I, _i64, _I]),
            "orc_tree_capacity": (_I, [_I, _I]),
            "orc_build_tree": (_I, [_I, _d, _I, _i64, _i64, _i64, _i64, _i64]),
            "orc_node_moments": (None, [_I, _i64, _i64, _i64, _d, _d, _d, _d, _d, _d, _d, _d, _d, _d, _d, _d,
                                        ctypes.c_int]),
            "orc_node_contractions": (None, [_I, _d, _d, _d, _d, _d]),
            "orc_far_velocity": (None, [ctypes.c_double] * 3 + [_d] * 6 + [ctypes.c_int, _d]),
            "orc_tree_velocity": (ctypes.c_int, [_I, _d, _d, _d, _d, _d, _d, ctypes.c_int, ctypes.c_int,
                                                 _i64, _i64, _i64, _i64, _i64, _d, _d, _d, _d, _d, _d, _d, _d, _d,
                                                 ctypes.c_double, ctypes.c_int, ctypes.c_double, _i64, _i64, _d, _i8,
                                                 _i64, ctypes.c_int]),
            "orc_positions": (None, [_I, _i64, _i64, _i64, _i64]),
            "orc_segment_geometry": (None, [_I, _d, _d, _d, _d, _d, _d, _d, _d]),
            "orc_morton_box": (ctypes.c_double, [_I, _d, _d]),
            "orc_morton_keys": (None, [_I, _d, _d, ctypes.c_double, _u64]),
            "orc_morton_sort": (None, [_I, _u64, _i64, _u64]),
            "orc_morton_tree": (_I, [_I, _u64, _I, _i64, _i64, _i64, _i64]),
        }
        for name, (restype, argtypes) in sig.items():
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _LIB.append(handle)
    return _LIB[0]


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64a(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _p(a, kind=_d):
    return a.ctypes.data_as(kind)


def pairs(points, starts, directions, lengths, gamma, radius, model, raise_singular=True):
    """``pair_velocity`` (vortex_numba.py:42-109) once per row: returns (u (k,3), flags int8)."""
    points, starts, directions = _f64(points), _f64(starts), _f64(directions)
    lengths, gamma, radius = _f64(lengths), _f64(gamma), _f64(radius)
    k = len(points)
    out = np.zeros((k, 3))
    flags = np.zeros(k, dtype=np.int8)
    lib().orc_pairs(k, _p(points), _p(starts), _p(directions), _p(lengths), _p(gamma), _p(radius), int(model),
                    int(bool(raise_singular)), _p(out), _p(flags, _i8))
    return out, flags


def exclusion_csr(point_count, pair_array):
    """vortex_numba.exclusion_csr (vortex_numba.py:228-243) for pairs whose points lie in range."""
    pair_array = _i64a(np.asarray(pair_array, dtype=np.int64).reshape(-1, 2))
    e = len(pair_array)
    ptr = np.zeros(point_count + 1, dtype=np.int64)
    if e == 0:
        return ptr, np.zeros(0, dtype=np.int64)
    seg = np.zeros(e, dtype=np.int64)
    count = lib().orc_exclusion_csr(point_count, e, _p(pair_array, _i64), _p(ptr, _i64), _p(seg, _i64))
    return ptr, seg[:count].copy()


def incident_pairs(nodes, edges, first):
    """network_numba.incident_pairs (network_numba.py:242-256) for (n,3) nodes and in-range (e,2) edges."""
    nodes = _f64(np.asarray(nodes, dtype=np.float64).reshape(-1, 3))
    edges = _i64a(np.asarray(edges, dtype=np.int64).reshape(-1, 2))
    n, e = len(nodes), len(edges)
    total = lib().orc_incident_pairs(n, _p(nodes), e, _p(edges, _i64), int(first), None, 0)
    pairs = np.zeros((total, 2), dtype=np.int64)
    if total:
        lib().orc_incident_pairs(n, _p(nodes), e, _p(edges, _i64), int(first), _p(pairs, _i64), total)
    return pairs


def direct_sum(points, starts, directions, lengths, gamma, radius, model, csr, singularity, threads=0,
               return_flags=False):
    """vortex_numba.direct_sum (vortex_numba.py:246-260): (velocity, any_flag)."""
    points, starts, directions = _f64(points), _f64(starts), _f64(directions)
    lengths, gamma, radius = _f64(lengths), _f64(gamma), _f64(radius)
    ptr, seg = _i64a(csr[0]), _i64a(csr[1])
    if len(seg) == 0:
        seg = np.zeros(1, dtype=np.int64)
    n, m = len(points), len(starts)
    out = np.zeros((n, 3))
    flags = np.zeros(n, dtype=np.int8)
    if n:
        lib().orc_direct_sum(n, _p(points), m, _p(starts), _p(directions), _p(lengths), _p(gamma), _p(radius),
                             int(model), int(singularity == "raise"), _p(ptr, _i64), _p(seg, _i64), _p(out),
                             _p(flags, _i8), int(threads))
    if return_flags:
        return out, flags
    return out, bool(np.any(flags))


def pair_matrix(points, starts, directions, lengths, radius, model, raise_singular=True):
    """vortex_numba.pair_matrix (vortex_numba.py:271-287): (pairs (n,m,3), flags (n,))."""
    points, starts, directions, lengths, radius = map(_f64, (points, starts, directions, lengths, radius))
    n, m = len(points), len(starts)
    out = np.zeros((n, m, 3))
    flags = np.zeros(n, dtype=np.int8)
    lib().orc_pair_matrix(n, _p(points), m, _p(starts), _p(directions), _p(lengths), _p(radius), int(model),
                          int(bool(raise_singular)), _p(out), _p(flags, _i8))
    return out, flags


def assemble_columns(pairs, column_ptr, column_segment, column_sign):
    """vortex_numba.assemble_columns (vortex_numba.py:290-308): out[p, j] = sum_k sign_k * pairs[p, segment_k],
    sequential in k from 0.0 (element-wise NumPy, the same IEEE operations per element)."""
    pairs = np.asarray(pairs, dtype=np.float64)
    out = np.zeros((pairs.shape[0], len(column_ptr) - 1, 3))
    for j in range(len(column_ptr) - 1):
        acc = np.zeros((pairs.shape[0], 3))
        for k in range(column_ptr[j], column_ptr[j + 1]):
            acc = acc + column_sign[k] * pairs[:, column_segment[k], :]
        out[:, j] = acc
    return out


def segment_geometry(starts, directions, lengths, gamma):
    """(length_vectors, ends, alpha, mid) exactly as vortex_tree.tree_sum forms them (vortex_tree.py:608-611)."""
    starts, directions, lengths, gamma = map(_f64, (starts, directions, lengths, gamma))
    m = len(starts)
    lv, ends, alpha, mid = (np.zeros((m, 3)) for _ in range(4))
    if m:
        lib().orc_segment_geometry(m, _p(starts), _p(directions), _p(lengths), _p(gamma), _p(lv), _p(ends),
                                   _p(alpha), _p(mid))
    return lv, ends, alpha, mid


def build_tree(mid, leaf_size):
    """vortex_tree.build_tree (vortex_tree.py:208-241): (order, lo, hi, left, right, count)."""
    mid = _f64(mid)
    n = len(mid)
    cap = lib().orc_tree_capacity(n, int(leaf_size))
    order = np.zeros(max(n, 1), dtype=np.int64)
    lo, hi, left, right = (np.zeros(cap, dtype=np.int64) for _ in range(4))
    count = lib().orc_build_tree(n, _p(mid), int(leaf_size), _p(order, _i64), _p(lo, _i64), _p(hi, _i64),
                                 _p(left, _i64), _p(right, _i64))
    return order[:n].copy(), lo[:count].copy(), hi[:count].copy(), left[:count].copy(), right[:count].copy(), count


def node_moments(order, lo, hi, starts, ends, alpha, length_vectors, radius, gamma, threads=0):
    """vortex_tree.node_moments (vortex_tree.py:309-376): (centre, bound, core, m0, m1, m2)."""
    order, lo, hi = _i64a(order), _i64a(lo), _i64a(hi)
    starts, ends, alpha, length_vectors, radius, gamma = map(_f64, (starts, ends, alpha, length_vectors, radius, gamma))
    count = len(lo)
    centre, m0 = np.zeros((count, 3)), np.zeros((count, 3))
    bound, core = np.zeros(count), np.zeros(count)
    m1, m2 = np.zeros((count, 3, 3)), np.zeros((count, 3, 3, 3))
    if count:
        lib().orc_node_moments(count, _p(order, _i64), _p(lo, _i64), _p(hi, _i64), _p(starts), _p(ends), _p(alpha),
                               _p(length_vectors), _p(radius), _p(gamma), _p(centre), _p(bound), _p(core), _p(m0),
                               _p(m1), _p(m2), int(threads))
    return centre, bound, core, m0, m1, m2


def node_contractions(m1, m2):
    """vortex_tree.node_contractions (vortex_tree.py:425-447): (w1, t2, w2)."""
    m1, m2 = _f64(m1), _f64(m2)
    count = len(m1)
    w1, t2, w2 = np.zeros((count, 3)), np.zeros((count, 3)), np.zeros((count, 3, 3))
    if count:
        lib().orc_node_contractions(count, _p(m1), _p(m2), _p(w1), _p(t2), _p(w2))
    return w1, t2, w2


def far_velocity(r, m0, m1, m2, w1, t2, w2, order):
    """vortex_tree.far_velocity (vortex_tree.py:450-497) for one node's arrays."""
    out = np.zeros(3)
    arrays = [_f64(a) for a in (m0, m1, m2, w1, t2, w2)]
    lib().orc_far_velocity(float(r[0]), float(r[1]), float(r[2]), *[_p(a) for a in arrays], int(order), _p(out))
    return out


def positions(ptr, seg, order):
    """vortex_tree._positions (vortex_tree.py:571-580): excluded segment ids as sorted tree positions."""
    ptr, seg, order = _i64a(ptr), _i64a(seg), _i64a(order)
    if len(seg) == 0:
        return seg
    inverse = np.empty_like(order)
    inverse[order] = np.arange(len(order))
    out = np.zeros_like(seg)
    lib().orc_positions(len(ptr) - 1, _p(ptr, _i64), _p(seg, _i64), _p(inverse, _i64), _p(out, _i64))
    return out


def tree_velocity(points, starts, directions, lengths, gamma, radius, model, singularity, tree, quantities, theta,
                  order, clearance, ex_ptr, ex_pos, threads=0):
    """vortex_tree.tree_velocity (vortex_tree.py:508-568) on any tree.

    ``tree`` = (order, lo, hi, left, right); ``quantities`` = (centre, bound, core, m0, m1, m2, w1, t2, w2).
    Returns (out, flags, far_counts, overflow)."""
    points, starts, directions, lengths, gamma, radius = map(_f64, (points, starts, directions, lengths, gamma,
                                                                    radius))
    t = [_i64a(a) for a in tree]
    q = [_f64(a) for a in quantities]
    ex_ptr = _i64a(ex_ptr)
    ex_pos = _i64a(ex_pos) if len(ex_pos) else np.zeros(1, dtype=np.int64)
    n = len(points)
    out = np.zeros((n, 3))
    flags = np.zeros(n, dtype=np.int8)
    far = np.zeros(n, dtype=np.int64)
    overflow = 0
    if n:
        overflow = lib().orc_tree_velocity(
            n, _p(points), _p(starts), _p(directions), _p(lengths), _p(gamma), _p(radius), int(model),
            int(singularity == "raise"), *[_p(a, _i64) for a in t], *[_p(a) for a in q], float(theta), int(order),
            float(clearance), _p(ex_ptr, _i64), _p(ex_pos, _i64), _p(out), _p(flags, _i8), _p(far, _i64),
            int(threads))
    return out, flags, far, bool(overflow)


def morton_tree(starts, directions, lengths, leaf_size):
    """CPU recomputation of the B200 Morton tree (morton_oracle.c): dict of keys, sorted keys, order, lo, hi, left,
    right, box, inv."""
    starts, directions, lengths = map(_f64, (starts, directions, lengths))
    m = len(starts)
    _, _, _, mid = segment_geometry(starts, directions, lengths, np.zeros(m))
    box = np.zeros(6)
    inv = lib().orc_morton_box(m, _p(mid), _p(box)) if m else 0.0
    keys = np.zeros(max(m, 1), dtype=np.uint64)
    order = np.zeros(max(m, 1), dtype=np.int64)
    sorted_keys = np.zeros(max(m, 1), dtype=np.uint64)
    if m:
        lib().orc_morton_keys(m, _p(mid), _p(box), inv, _p(keys, _u64))
        lib().orc_morton_sort(m, _p(keys, _u64), _p(order, _i64), _p(sorted_keys, _u64))
    cap = max(2 * m, 1)
    lo, hi, left, right = (np.zeros(cap, dtype=np.int64) for _ in range(4))
    count = lib().orc_morton_tree(m, _p(sorted_keys, _u64), int(leaf_size), _p(lo, _i64), _p(hi, _i64),
                                  _p(left, _i64), _p(right, _i64))
    return dict(keys=keys[:m].copy(), sorted_keys=sorted_keys[:m].copy(), order=order[:m].copy(), lo=lo[:count].copy(),
                hi=hi[:count].copy(), left=left[:count].copy(), right=right[:count].copy(), box=box, inv=inv,
                count=count)


def tree_sum(points, starts, directions, lengths, gamma, radius, model, csr, singularity, theta=0.5, order=2,
             leaf_size=32, core_clearance=3.0, kind="median", threads=0, details=False):
    """vortex_tree.tree_sum (vortex_tree.py:588-626): (velocity, any_flag).

    ``kind='median'`` builds the reference's median-split tree; ``kind='morton'`` the B200 build's Morton tree (its CPU
    recomputation), evaluated with the reference's traversal.  ``details=True`` adds a dict with the tree, node
    quantities, flags and far counts."""
    if int(model) not in SUPPORTED_TREE_MODELS and np.any(np.asarray(radius) > 0):
        raise ValueError("tree backend supports core models NONE, RANKINE and LAMB_OSEEN only")
    if theta >= 1.0:
        raise ValueError("tree theta must be below one")
    points, starts, directions, lengths, gamma, radius = map(_f64, (points, starts, directions, lengths, gamma,
                                                                    radius))
    n, m = len(points), len(starts)
    if n == 0 or m == 0:
        out = np.zeros((n, 3))
        return (out, False, {}) if details else (out, False)
    lv, ends, alpha, mid = segment_geometry(starts, directions, lengths, gamma)
    if kind == "median":
        tree = build_tree(mid, leaf_size)[:5]
    elif kind == "morton":
        mt = morton_tree(starts, directions, lengths, leaf_size)
        tree = (mt["order"], mt["lo"], mt["hi"], mt["left"], mt["right"])
    else:
        raise ValueError(kind)
    centre, bound, core, m0, m1, m2 = node_moments(tree[0], tree[1], tree[2], starts, ends, alpha, lv, radius, gamma,
                                                   threads)
    w1, t2, w2 = node_contractions(m1, m2)
    ex_pos = positions(csr[0], csr[1], tree[0])
    quantities = (centre, bound, core, m0, m1, m2, w1, t2, w2)
    out, flags, far, overflow = tree_velocity(points, starts, directions, lengths, gamma, radius, model, singularity,
                                              tree, quantities, theta, order, core_clearance, csr[0], ex_pos, threads)
    if overflow:
        raise RuntimeError("tree traversal stack overflow on the CPU oracle")
    if details:
        return out, bool(np.any(flags)), dict(tree=tree, quantities=quantities, flags=flags, far=far, ex_pos=ex_pos)
    return out, bool(np.any(flags))
