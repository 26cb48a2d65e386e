"""B200-native free-wake induced-velocity hot path (regularised Biot-Savart direct sum and Barnes-Hut tree code).

Drop-in modules for the reference's GPU vortex backends: ``openfawe_b200.vortex_cuda`` (``cuda_sum``) and
``openfawe_b200.vortex_cuda_tree`` (``cuda_tree_sum``); ``openfawe_b200.install()`` registers them under the
reference's module names so that ``segments_velocity(..., backend='cuda'|'cuda_tree')`` reaches them unchanged.
"""
from .settings import CoreModel, CudaSettings, TreeSettings  # noqa: F401


def install(package="openfawe.aero", **options):
    """Register the drop-in modules as ``<package>.vortex_cuda`` and ``<package>.vortex_cuda_tree``; keyword options
    (tree, order, theta, leaf_size) as in ``openfawe_b200.dropin.install``."""
    from .dropin import install as _install
    return _install(package, **options)


def uninstall(package="openfawe.aero"):
    """Undo ``install``."""
    from .dropin import uninstall as _uninstall
    _uninstall(package)
