"""The drop-in modules for the reference's GPU build and GPU node quantities (vortex_cuda_build.device_build_tree,
vortex_cuda_moments.device_node_quantities / node_quantities) against the reference's CPU arrays: the tree element for
element (its GPU build's contract, tests/test_cuda_build.py of the reference), centre / core / bound bit for bit and
moments within 1e-12 node-relative (tests/test_cuda_moments.py:90-105 of the reference), repeatable bit for bit."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def node_relative(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.abs(a).reshape(len(a), -1).max(axis=1)
    diff = np.abs(a - b).reshape(len(a), -1).max(axis=1)
    return np.where(scale > 0, diff / np.where(scale > 0, scale, 1.0), diff)


def test_device_build_tree_element_for_element(device):
    from openfawe_b200 import vortex_cuda_build as VCB
    g = golden("tree_build.npz")
    names = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_mid")})
    assert names
    VCB.Statistics.reset_totals()
    for name in names:
        mid, leaf = g[f"{name}_mid"], int(g[f"{name}_leaf"])
        d_order, order, lo, hi, left, right, count = VCB.device_build_tree(mid, leaf)
        for key, value in zip(("order", "lo", "hi", "left", "right"), (order, lo, hi, left, right)):
            assert np.array_equal(value, g[f"{name}_{key}"]), (name, key)
        assert count == len(g[f"{name}_lo"])
        assert np.array_equal(d_order.copy_to_host(), order)
    assert VCB.Statistics.totals["calls"] == len(names)
    # no midpoints: one empty leaf
    _, order, lo, hi, left, right, count = VCB.device_build_tree(np.zeros((0, 3)), 8)
    assert count == 1 and list(lo) == [0] and list(hi) == [0] and list(left) == [-1] and list(right) == [-1]


def test_node_quantities_against_reference(device):
    from openfawe_b200 import vortex_cuda_moments as VCM
    g = golden("moments.npz")
    for seed in (1, 2, 3):
        p = lambda k: g[f"s{seed}_{k}"]  # noqa: E731
        lv = p("directions") * p("lengths")[:, None]
        ends = p("starts") + lv
        alpha = p("gamma")[:, None] * lv
        args = (p("order"), p("lo"), p("hi"), p("starts"), ends, alpha, lv, p("radius"), p("gamma"))
        got = dict(zip(VCM.QUANTITIES, VCM.node_quantities(*args)))
        for key in ("centre", "core", "bound"):
            assert np.array_equal(got[key], p(key)), (seed, key)
        for key in ("m0", "m1", "m2"):
            assert node_relative(p(key), got[key]).max() <= 1e-12, (seed, key)
        for key, made_of in (("w1", "m1"), ("t2", "m2"), ("w2", "m2")):
            scale = np.abs(p(made_of)).reshape(len(p(made_of)), -1).max(axis=1)
            diff = np.abs(p(key) - got[key]).reshape(len(got[key]), -1).max(axis=1)
            assert np.all(diff <= 1e-12 * scale), (seed, key)
        again = VCM.node_quantities(*args)
        assert all(np.array_equal(a, got[k]) for k, a in zip(VCM.QUANTITIES, again))
        single = VCM.device_node_quantities(*args, single=True)
        assert single["m2"].dtype == np.float32 and np.array_equal(single["m2_64"].copy_to_host(), got["m2"])
        with pytest.raises(ValueError):
            VCM.device_node_quantities(*args[:5], 2.0 * alpha, *args[6:])
