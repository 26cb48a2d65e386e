"""Make the reference's callers reach this library unchanged.

``segments_velocity`` imports its GPU backends lazily inside the call (``from .vortex_cuda import cuda_sum``,
``from .vortex_cuda_tree import cuda_tree_sum``; src/openfawe/aero/vortex.py:476-483, and ``available`` /
``probe_error`` at vortex.py:119-134).  Python resolves those relative imports through ``sys.modules`` first, so
registering this package's modules under the reference's names swaps the backends without editing any caller
(VSM, lifting line, lattice, wake convection, flight loop).
"""
import sys


def install(package="openfawe.aero"):
    """Register ``openfawe_b200.vortex_cuda`` / ``vortex_cuda_tree`` as ``<package>.vortex_cuda`` / ``..._tree``.

    Returns the two modules.  Call it before the first GPU-backend call of the process (or after, since the reference
    imports them inside each call)."""
    from . import vortex_cuda, vortex_cuda_tree
    sys.modules[package + ".vortex_cuda"] = vortex_cuda
    sys.modules[package + ".vortex_cuda_tree"] = vortex_cuda_tree
    parent = sys.modules.get(package)
    if parent is not None:
        setattr(parent, "vortex_cuda", vortex_cuda)
        setattr(parent, "vortex_cuda_tree", vortex_cuda_tree)
    return vortex_cuda, vortex_cuda_tree


def uninstall(package="openfawe.aero"):
    """Remove the registrations made by ``install``."""
    for name in ("vortex_cuda", "vortex_cuda_tree"):
        module = sys.modules.get(f"{package}.{name}")
        if module is not None and module.__name__.startswith("openfawe_b200."):
            del sys.modules[f"{package}.{name}"]
            parent = sys.modules.get(package)
            if parent is not None and getattr(parent, name, None) is module:
                delattr(parent, name)
