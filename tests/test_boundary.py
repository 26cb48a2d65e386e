"""The drop-in boundary without a GPU: the C-ABI library loads and exports every declared entry point, the Python
mirrors of the reference's settings validate like the reference's, and the modules register under the reference's
names.  No compute call is made here."""
import ctypes
import os
import re
import sys

import numpy as np
import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "bs_b200.h")


def declared_functions():
    text = open(HEADER, encoding="utf-8").read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from openfawe_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared_functions()
    assert "bs_direct" in names and "bs_tree_eval" in names and len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    from openfawe_b200 import _lib
    assert set(_lib.SIGNATURES) <= set(names)
    major, minor, arch = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert lib.bs_version(ctypes.byref(major), ctypes.byref(minor), ctypes.byref(arch)) == 0
    assert arch.value == 100


def test_struct_layouts_match_header():
    from openfawe_b200 import _lib
    assert ctypes.sizeof(_lib.Sources) == 48
    assert ctypes.sizeof(_lib.Targets) == 40
    assert ctypes.sizeof(_lib.KernelParams) == 24
    assert ctypes.sizeof(_lib.TreeParams) == 40
    assert _lib.TreeParams.stack_limit.offset == 36


def test_settings_mirror_reference_validation():
    from openfawe_b200.settings import CudaSettings, TreeSettings
    for bad in (dict(theta=1.0), dict(theta=0.0), dict(order=3), dict(leaf_size=0), dict(core_clearance=-1.0),
                dict(theta=True)):
        with pytest.raises(ValueError):
            TreeSettings(**bad)
    for bad in (dict(precision="fp16"), dict(block=48), dict(block=True), dict(suspect="gpu"),
                dict(precision="fp64", suspect="gpu64"), dict(moments="device"), dict(build="device"),
                dict(tree="octree"), dict(near=-1.0)):
        with pytest.raises(ValueError):
            CudaSettings(**bad)
    assert CudaSettings().precision == "mixed" and CudaSettings().tree == "median"


def test_install_registers_reference_module_names():
    import openfawe_b200
    vc, vct = openfawe_b200.install("fakepkg.aero")
    try:
        assert sys.modules["fakepkg.aero.vortex_cuda"] is vc
        assert sys.modules["fakepkg.aero.vortex_cuda_tree"] is vct
        for name in ("cuda_sum", "available", "probe_error", "Statistics"):
            assert hasattr(vc, name)
        assert hasattr(vct, "cuda_tree_sum") and hasattr(vct, "Statistics")
    finally:
        openfawe_b200.uninstall("fakepkg.aero")
    assert "fakepkg.aero.vortex_cuda" not in sys.modules


def test_no_device_means_value_error_not_fallback(monkeypatch):
    """Without a usable device the backends refuse, like the reference's (vortex_cuda.py:384-385)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from openfawe_b200 import vortex_cuda, vortex_cuda_tree
    from openfawe_b200.settings import CudaSettings, TreeSettings
    monkeypatch.setattr(vortex_cuda, "_AVAILABLE", [])
    monkeypatch.setattr(vortex_cuda, "_PROBE_ERROR", [])
    args = (np.zeros((1, 3)), np.zeros((1, 3)), np.array([[1.0, 0, 0]]), np.ones(1), np.ones(1), np.zeros(1), 0,
            (np.zeros(2, dtype=np.int64), np.zeros(0, dtype=np.int64)), "raise")
    with pytest.raises(ValueError, match="needs a CUDA device"):
        vortex_cuda.cuda_sum(*args, CudaSettings("fp64"))
    with pytest.raises(ValueError, match="needs a CUDA device"):
        vortex_cuda_tree.cuda_tree_sum(*args, TreeSettings(), CudaSettings("fp64"))
    assert vortex_cuda.probe_error()


def test_product_never_imports_the_oracle():
    """The oracle is the checker only: no module of the package imports it."""
    pkg = os.path.join(REPO, "openfawe_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                text = open(os.path.join(root, f), encoding="utf-8").read()
                assert "import oracle" not in text and "from oracle" not in text, f


def test_wake_generators_shapes():
    from openfawe_b200 import wakes
    c1 = wakes.lattice()
    assert len(c1["starts"]) == 4207 and len(c1["points"]) == 1024 and c1["model"] == 5
    c2 = wakes.rotor_sheet(468)
    assert len(c2["starts"]) == 219 * 468 - 46 and len(c2["points"]) == 20570 and c2["model"] == 2
    s = wakes.selftest_sheet(468, seed=468)
    assert len(s["starts"]) == 102382 and len(s["points"]) == 20570


def test_install_registers_build_and_moments_modules_and_patches_functions():
    import types
    import openfawe_b200
    from openfawe_b200 import dropin, network, operators
    openfawe_b200.install("fakepkg2.aero")
    try:
        assert sys.modules["fakepkg2.aero.vortex_cuda_moments"].__name__ == "openfawe_b200.vortex_cuda_moments"
        assert sys.modules["fakepkg2.aero.vortex_cuda_build"].__name__ == "openfawe_b200.vortex_cuda_build"
    finally:
        openfawe_b200.uninstall("fakepkg2.aero")
    assert "fakepkg2.aero.vortex_cuda_build" not in sys.modules
    # stand-ins for the reference's compiled modules, already imported
    fakes = {name: types.ModuleType(name) for name in ("fk.aero.network_numba", "fk.aero.vortex_numba",
                                                       "fk.rotor.ring_wake")}
    originals = {}
    for name, module in fakes.items():
        for fn in ("incident_pairs", "exclusion_csr", "pair_matrix", "assemble_columns"):
            original = (lambda *a: None)
            setattr(module, fn, original)
            originals[(name, fn)] = original
        sys.modules[name] = module
    try:
        saved = dropin.patch_functions("fk")
        assert fakes["fk.aero.network_numba"].incident_pairs is network.incident_pairs
        assert fakes["fk.rotor.ring_wake"].incident_pairs is network.incident_pairs
        assert fakes["fk.aero.vortex_numba"].exclusion_csr is network.exclusion_csr
        assert fakes["fk.aero.vortex_numba"].pair_matrix is operators.pair_matrix
        assert fakes["fk.aero.vortex_numba"].assemble_columns is operators.assemble_columns
        # names this library does not replace stay as they were
        assert fakes["fk.aero.network_numba"].exclusion_csr is originals[("fk.aero.network_numba", "exclusion_csr")]
        dropin.unpatch_functions(saved)
        assert fakes["fk.aero.vortex_numba"].pair_matrix is originals[("fk.aero.vortex_numba", "pair_matrix")]
    finally:
        for name in fakes:
            del sys.modules[name]


def test_install_options_map_reference_settings():
    """install(...) options reach calls whose settings cannot express them, and record what they change."""
    from conftest import ReferenceCudaSettings, ReferenceTreeSettings
    import openfawe_b200
    from openfawe_b200 import vortex_cuda_tree as VCT
    from openfawe_b200.settings import CudaSettings
    tree, cuda = ReferenceTreeSettings(theta=0.04), ReferenceCudaSettings()
    try:
        assert VCT.effective(tree, cuda) == ("median", 2, 0.04, 32)
        openfawe_b200.install("openfawe_b200_test_pkg", tree="morton", order=5, theta={0.04: 0.215}, leaf_size=384)
        assert VCT.effective(tree, cuda) == ("morton", 5, 0.215, 384)
        # thetas outside the dict are kept; an explicit tree field and the order= keyword win
        assert VCT.effective(ReferenceTreeSettings(theta=0.2), cuda) == ("morton", 5, 0.2, 384)
        assert VCT.effective(tree, CudaSettings(tree="median"), order=3) == ("median", 3, 0.215, 384)
        VCT.configure(theta=lambda t: 5 * t)
        assert VCT.effective(tree, cuda) == ("median", 2, 0.2, 32)
        VCT.configure(theta=0.3)
        assert VCT.effective(tree, cuda)[2] == 0.3
        for bad in (dict(tree="octree"), dict(order=6), dict(leaf_size=0), dict(theta=1.5)):
            with pytest.raises(ValueError):
                VCT.configure(**bad)
    finally:
        openfawe_b200.uninstall("openfawe_b200_test_pkg")
    assert VCT.OPTIONS == {} and VCT.effective(tree, cuda) == ("median", 2, 0.04, 32)
