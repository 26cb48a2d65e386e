"""ctypes binding of libbs_b200.so (include/bs_b200.h) and the per-device context.

The library is the only compute path: when it is missing or cannot initialise a device, every entry point raises;
nothing falls back to the CPU.  ctypes releases the GIL for the duration of each C call.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libbs_b200.so")

BS_OK, BS_ERR_ARG, BS_ERR_CUDA, BS_ERR_STACK, BS_ERR_TIMEOUT, BS_ERR_OOM = range(6)
BS_FP64, BS_MIXED, BS_FP32 = range(3)
BS_TREE_MEDIAN, BS_TREE_MORTON = range(2)

_p = ctypes.c_void_p
_i64 = ctypes.c_int64


class Sources(ctypes.Structure):
    _fields_ = [("m", _i64), ("starts", _p), ("directions", _p), ("lengths", _p), ("gamma", _p), ("radius", _p)]


class Targets(ctypes.Structure):
    _fields_ = [("n", _i64), ("points", _p), ("ex_ptr", _p), ("ex_seg", _p), ("e", _i64)]


class KernelParams(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int), ("raise_singular", ctypes.c_int), ("precision", ctypes.c_int),
                ("block", ctypes.c_int), ("near_cores", ctypes.c_double)]


class TreeParams(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_double), ("order", ctypes.c_int), ("leaf_size", _i64),
                ("clearance", ctypes.c_double), ("kind", ctypes.c_int), ("stack_limit", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("points", _i64), ("segments", _i64), ("nodes", _i64), ("launches", _i64),
                ("far_evaluations", _i64), ("near_pairs", _i64), ("fp64_pairs", _i64), ("visits", _i64),
                ("build_ms", ctypes.c_double), ("moments_ms", ctypes.c_double), ("evaluate_ms", ctypes.c_double),
                ("pair_slots", _i64), ("walk_ms", ctypes.c_double), ("list_ms", ctypes.c_double),
                ("upload_ms", ctypes.c_double), ("download_ms", ctypes.c_double), ("far_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


SIGNATURES = {
    "bs_init": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_p)]),
    "bs_destroy": (None, [_p]),
    "bs_last_error": (ctypes.c_char_p, []),
    "bs_last_stats": (ctypes.c_int, [_p, ctypes.POINTER(Stats)]),
    "bs_version": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)] * 3),
    "bs_fp32_peak": (ctypes.c_int, [_p, ctypes.POINTER(ctypes.c_double)]),
    "bs_upload": (ctypes.c_int, [_p, _p, _p, ctypes.c_size_t, _p]),
    "bs_upload_many": (ctypes.c_int, [_p, ctypes.c_int, _p, _p, _p, _p]),
    "bs_download_many": (ctypes.c_int, [_p, ctypes.c_int, _p, _p, _p, _p]),
    "bs_tree_sum_host": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.POINTER(TreeParams),
                                        ctypes.POINTER(Targets), ctypes.POINTER(KernelParams), _p, _p, _p, _p]),
    "bs_direct": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.POINTER(Targets), ctypes.POINTER(KernelParams),
                                 _p, _p, _p]),
    "bs_tree_build": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.POINTER(TreeParams), ctypes.POINTER(_p),
                                     _p]),
    "bs_tree_from_arrays": (ctypes.c_int, [_p, ctypes.POINTER(Sources), _p, _p, _p, _p, _p, _i64,
                                           ctypes.POINTER(_p), _p]),
    "bs_tree_free": (None, [_p]),
    "bs_tree_count": (_i64, [_p]),
    "bs_tree_export": (ctypes.c_int, [_p] * 15 + [_p]),
    "bs_tree_keys": (ctypes.c_int, [_p, _p, _p, _p]),
    "bs_tree_eval": (ctypes.c_int, [_p, _p, ctypes.POINTER(TreeParams), ctypes.POINTER(Targets),
                                    ctypes.POINTER(KernelParams), _p, _p, _p, _p]),
    "bs_tree_sum": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.POINTER(TreeParams), ctypes.POINTER(Targets),
                                   ctypes.POINTER(KernelParams), _p, _p, _p, _p]),
    "bs_forest_build": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.c_int, _p, ctypes.POINTER(TreeParams),
                                       ctypes.POINTER(_p), _p]),
    "bs_forest_roots": (ctypes.c_int, [_p, _p, _p]),
    "bs_forest_eval": (ctypes.c_int, [_p, _p, ctypes.POINTER(TreeParams), ctypes.POINTER(Targets), _p,
                                      ctypes.POINTER(KernelParams), _p, _p, _p, _p]),
    "bs_forest_graph": (ctypes.c_int, [_p, _p, ctypes.POINTER(TreeParams), ctypes.POINTER(Targets), _p,
                                       ctypes.POINTER(KernelParams), _p, _p, _p, ctypes.POINTER(_p)]),
    "bs_forest_eval_exact": (ctypes.c_int, [_p, _p, ctypes.POINTER(TreeParams), ctypes.POINTER(Targets), _p, _p,
                                            ctypes.POINTER(KernelParams), _p, _p, _p, _p]),
    "bs_forest_graph_exact": (ctypes.c_int, [_p, _p, ctypes.POINTER(TreeParams), ctypes.POINTER(Targets), _p, _p,
                                             ctypes.POINTER(KernelParams), _p, _p, _p, ctypes.POINTER(_p)]),
    "bs_graph_launch": (ctypes.c_int, [_p, _p]),
    "bs_graph_status": (ctypes.c_int, [_p, ctypes.POINTER(Stats)]),
    "bs_graph_free": (None, [_p]),
    "bs_incident_pairs": (ctypes.c_int, [_p, _p, ctypes.c_int64, _p, ctypes.c_int64, ctypes.c_int64, _p, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int64), _p]),
    "bs_exclusion_csr": (ctypes.c_int, [_p, ctypes.c_int64, _p, ctypes.c_int64, _p, _p, ctypes.POINTER(ctypes.c_int64),
                                        _p]),
    "bs_tree_adjoint": (ctypes.c_int, [_p, ctypes.POINTER(Sources), ctypes.POINTER(TreeParams),
                                       ctypes.POINTER(Targets), ctypes.POINTER(KernelParams)] + [_p] * 6),
    "bs_median_topology": (ctypes.c_int, [_p, ctypes.c_int64, _p, ctypes.c_int, _p, _p, _p, _p, _p, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int64), _p]),
    "bs_node_quantities": (ctypes.c_int, [_p, ctypes.c_int64, _p, _p, _p, _p, _p, ctypes.c_int64, _p, _p, _p]
                           + [_p] * 9 + [_p]),
    "bs_pair_matrix": (ctypes.c_int, [_p, ctypes.c_int64, _p, ctypes.POINTER(Sources), ctypes.c_int, ctypes.c_int, _p,
                                      _p, _p]),
    "bs_assemble_columns": (ctypes.c_int, [_p, ctypes.c_int64, ctypes.c_int64, _p, ctypes.c_int64, _p, _p, _p, _p,
                                           _p]),
    "bs_ring_columns": (ctypes.c_int, [_p, ctypes.c_int64, _p, ctypes.POINTER(Sources), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int64, _p, _p, _p, _p, _p, _p]),
}

_LOCK = threading.RLock()
_LIB = []
_CONTEXTS = {}


def library():
    """The loaded library (raises RuntimeError when the shared object is missing)."""
    if not _LIB:
        with _LOCK:
            if not _LIB:
                if not os.path.exists(LIBRARY):
                    raise RuntimeError(f"{LIBRARY} is missing: build it with `python -m openfawe_b200.build` "
                                       "(there is no CPU fallback)")
                lib = ctypes.CDLL(LIBRARY)
                for name, (restype, argtypes) in SIGNATURES.items():
                    fn = getattr(lib, name)
                    fn.restype = restype
                    fn.argtypes = argtypes
                _LIB.append(lib)
    return _LIB[0]


def last_error():
    return library().bs_last_error().decode(errors="replace")


class StackOverflow(RuntimeError):
    pass


def check(status, what):
    """Map a bs_status to the exception the reference raises in the same situation."""
    if status == BS_OK:
        return
    text = f"{what}: {last_error()}"
    if status == BS_ERR_ARG:
        raise ValueError(text)
    if status == BS_ERR_STACK:
        raise StackOverflow(text)
    if status == BS_ERR_OOM:
        raise MemoryError(text)
    raise RuntimeError(text)


def context(device=0):
    """The library context of a device (created on first use; raises when the device cannot be used)."""
    device = int(device)
    if device not in _CONTEXTS:
        with _LOCK:
            if device not in _CONTEXTS:
                handle = _p()
                check(library().bs_init(device, ctypes.byref(handle)), f"bs_init(device={device})")
                _CONTEXTS[device] = handle
    return _CONTEXTS[device]


def stats(device=0):
    s = Stats()
    check(library().bs_last_stats(context(device), ctypes.byref(s)), "bs_last_stats")
    return s.as_dict()
