"""Configuration types of the vortex-batch backends, mirroring the reference's.

``CoreModel``, ``TreeSettings`` and ``CudaSettings`` repeat src/openfawe/aero/vortex.py:21-27, :30-55 and :58-116
(same fields, defaults and refusals), so a caller of the reference can pass either the reference's objects or these.
The backend functions read settings by attribute only (duck typing), and read the B200-only fields with ``getattr``
and a default, so the reference's frozen dataclasses work unchanged.

B200-only fields of ``CudaSettings`` (defaults keep the reference's behaviour):

* ``tree``: ``'median'`` (default) builds, on the GPU, the reference's median-split tree element for element
  (vortex_tree.build_tree), so that results match the reference's tree code; ``'morton'`` builds this library's
  Morton-key tree (GPU radix sort + binary radix tree), faster to build and used by the benchmarks.
* ``near``: core radii within which single-precision pairs are evaluated again in FP64 (default 3.0).
"""
from dataclasses import dataclass
from enum import IntEnum
import operator

import numpy as np


class CoreModel(IntEnum):
    NONE = 0
    RANKINE = 1
    LAMB_OSEEN = 2
    VATISTAS = 3
    OFFSET = 4
    ROSENHEAD_MOORE = 5


@dataclass(frozen=True)
class TreeSettings:
    """Barnes-Hut settings (vortex.py:30-55): opening ratio, expansion order 0-2, leaf size, core clearance."""
    theta: float = 0.5
    order: int = 2
    leaf_size: int = 32
    core_clearance: float = 3.0

    def __post_init__(self):
        if isinstance(self.theta, (bool, np.bool_)) or not (0 < float(self.theta) < 1):
            raise ValueError("tree theta must lie strictly between 0 and 1")
        if isinstance(self.order, (bool, np.bool_)) or self.order not in (0, 1, 2):
            raise ValueError("tree order must be 0, 1 or 2")
        if isinstance(self.leaf_size, (bool, np.bool_)) or operator.index(self.leaf_size) < 1:
            raise ValueError("tree leaf size must be a positive integer")
        if not np.isfinite(self.core_clearance) or self.core_clearance < 0:
            raise ValueError("tree core clearance must be finite and nonnegative")


@dataclass(frozen=True)
class CudaSettings:
    """GPU settings (vortex.py:58-116) plus the B200-only ``tree`` and ``near`` fields (module docstring).

    precision: 'fp64' (double throughout), 'mixed' (FP32 pair and far-field arithmetic on compensated two-float
    coordinates, FP64 near field and FP64 per-target sums) or 'fp32' (as mixed with FP32 per-target sums).
    block: threads per block (32, 64, 128 or 256).  suspect/control/moments/build/rings keep the reference's meaning
    and values; there is no CPU recomputation here, so 'cpu' and 'gpu64' both re-evaluate suspect pairs in FP64 on the
    GPU, and moments and build always run on the GPU.
    """
    precision: str = "mixed"
    block: int = 128
    suspect: str = "cpu"
    control: str = "cpu"
    moments: str = "cpu"
    build: str = "cpu"
    rings: str = "cpu"
    tree: str = "median"
    near: float = 3.0

    def __post_init__(self):
        if self.precision not in ("fp64", "mixed", "fp32"):
            raise ValueError("cuda precision must be 'fp64', 'mixed' or 'fp32'")
        if isinstance(self.block, (bool, np.bool_)) or self.block not in (32, 64, 128, 256):
            raise ValueError("cuda block must be 32, 64, 128 or 256")
        if self.suspect not in ("cpu", "gpu64"):
            raise ValueError("cuda suspect must be 'cpu' or 'gpu64'")
        if self.suspect == "gpu64" and self.precision == "fp64":
            raise ValueError("cuda suspect='gpu64' is for the single precisions 'mixed' and 'fp32' only")
        if self.control not in ("cpu", "gpu"):
            raise ValueError("cuda control must be 'cpu' or 'gpu'")
        if self.moments not in ("cpu", "gpu"):
            raise ValueError("cuda moments must be 'cpu' or 'gpu'")
        if self.build not in ("cpu", "gpu"):
            raise ValueError("cuda build must be 'cpu' or 'gpu'")
        if self.rings not in ("cpu", "gpu"):
            raise ValueError("cuda rings must be 'cpu' or 'gpu'")
        if self.tree not in ("median", "morton"):
            raise ValueError("cuda tree must be 'median' or 'morton'")
        if not np.isfinite(self.near) or self.near < 0:
            raise ValueError("cuda near must be finite and nonnegative")


PRECISION_CODES = {"fp64": 0, "mixed": 1, "fp32": 2}
TREE_KINDS = {"median": 0, "morton": 1}
