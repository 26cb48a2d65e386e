"""Make the reference's callers reach this library unchanged.

``segments_velocity`` imports its GPU backends lazily inside the call (``from .vortex_cuda import cuda_sum``,
``from .vortex_cuda_tree import cuda_tree_sum``; src/openfawe/aero/vortex.py:476-483, and ``available`` /
``probe_error`` at vortex.py:119-134).  Python resolves those relative imports through ``sys.modules`` first, so
registering this package's modules under the reference's names swaps the backends without editing any caller
(VSM, lifting line, lattice, wake convection, flight loop).
"""
import sys


def install(package="openfawe.aero", *, tree=None, order=None, theta=None, leaf_size=None):
    """Register ``openfawe_b200.vortex_cuda`` / ``vortex_cuda_tree`` / ``vortex_cuda_moments`` / ``vortex_cuda_build``
    under ``<package>``.

    Returns the two modules.  Call it before the first GPU-backend call of the process (or after, since the reference
    imports them inside each call).

    The keyword options reach the tree path through settings objects the caller cannot change (the reference's
    TreeSettings refuses orders above 2, its CudaSettings has no tree field): ``tree`` ('median' or 'morton'),
    ``order`` (0-5), ``theta`` (a number, a dict {caller's theta: theta} or a callable) and ``leaf_size`` apply to
    every later ``cuda_tree_sum`` call (``vortex_cuda_tree.configure``).  They change the approximation the caller
    asked for -- for example ``install(tree='morton', order=5, theta={0.04: 0.215}, leaf_size=384)`` swaps the
    order-2 tree at theta 0.04 for the fifth-order tree at the same error level -- and each call records what it
    ran in ``Statistics.last['effective']``.  Without options nothing changes."""
    from . import vortex_cuda, vortex_cuda_build, vortex_cuda_moments, vortex_cuda_tree
    vortex_cuda_tree.configure(tree=tree, order=order, theta=theta, leaf_size=leaf_size)
    modules = dict(vortex_cuda=vortex_cuda, vortex_cuda_tree=vortex_cuda_tree, vortex_cuda_moments=vortex_cuda_moments,
                   vortex_cuda_build=vortex_cuda_build)
    parent = sys.modules.get(package)
    for name, module in modules.items():
        sys.modules[f"{package}.{name}"] = module
        if parent is not None:
            setattr(parent, name, module)
    return vortex_cuda, vortex_cuda_tree


def uninstall(package="openfawe.aero"):
    """Remove the registrations made by ``install`` and clear its options."""
    from . import vortex_cuda_tree
    vortex_cuda_tree.configure()
    for name in ("vortex_cuda", "vortex_cuda_tree", "vortex_cuda_moments", "vortex_cuda_build"):
        module = sys.modules.get(f"{package}.{name}")
        if module is not None and module.__name__.startswith("openfawe_b200."):
            del sys.modules[f"{package}.{name}"]
            parent = sys.modules.get(package)
            if parent is not None and getattr(parent, name, None) is module:
                delattr(parent, name)


# Functions of the reference's compiled bookkeeping modules that this library replaces one for one, with the modules
# that bind them by name (ring_wake imports incident_pairs at import time, src/openfawe/rotor/ring_wake.py:17).
FUNCTIONS = {
    "aero.network_numba": {"incident_pairs": ("network", "incident_pairs")},
    "aero.vortex_numba": {"exclusion_csr": ("network", "exclusion_csr"),
                          "pair_matrix": ("operators", "pair_matrix"),
                          "assemble_columns": ("operators", "assemble_columns")},
    "rotor.ring_wake": {"incident_pairs": ("network", "incident_pairs")},
}


def patch_functions(root="openfawe"):
    """Point the already-imported reference modules' ``incident_pairs``, ``exclusion_csr``, ``pair_matrix`` and
    ``assemble_columns`` at this library's GPU versions (same signatures and results).  Modules not imported yet are
    skipped (import them first).  Returns the replaced originals for ``unpatch_functions``."""
    import importlib
    saved = []
    for module_name, names in FUNCTIONS.items():
        module = sys.modules.get(f"{root}.{module_name}")
        if module is None:
            continue
        for name, (ours, attr) in names.items():
            if hasattr(module, name):
                saved.append((module, name, getattr(module, name)))
                setattr(module, name, getattr(importlib.import_module(f"{__package__}.{ours}"), attr))
    return saved


def unpatch_functions(saved):
    """Restore what ``patch_functions`` replaced."""
    for module, name, original in reversed(saved):
        setattr(module, name, original)
