"""Unit-circulation influence operators on the GPU (bs_pair_matrix, bs_assemble_columns, bs_ring_columns) against the
reference's pair_matrix / assemble_columns outputs and the oracle.

Bounds: per-point flags identical; each pair within 1e-12 * sum_s |u_s| of its point (the reference's A1 bound of the
direct sum, applied to every term); assemble_columns bit for bit given the same pairs (its sums run in the reference's
order); the fused ring columns within the same 1e-12 bound.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def within_a1(got, ref):
    scale = np.linalg.norm(ref, axis=-1).sum(axis=1)  # sum_s |u_s| per point
    err = np.linalg.norm(got - ref, axis=-1)
    assert np.all(err <= 1e-12 * scale[:, None] + 1e-300), float(np.max(err / np.maximum(scale[:, None], 1e-300)))


def test_operators_match_reference_fixtures(device):
    from openfawe_b200 import operators, wakes
    g = golden("operators.npz")
    wing = wakes.ring_wing(panels=16, rows=3)
    layout = (wing["column_ptr"], wing["column_segment"], wing["column_sign"])
    points = g["points"]
    for model in (0, 2, 5):
        radius = wing["radius"] if model else np.zeros(len(wing["radius"]))
        for mode in ("raise", "zero"):
            key = f"m{model}_{mode}"
            pairs = np.full((len(points), len(wing["starts"]), 3), np.nan)
            flags = np.full(len(points), 9, dtype=np.int8)
            operators.pair_matrix(points, wing["starts"], wing["directions"], wing["lengths"], radius, model,
                                  mode == "raise", pairs, flags, device)
            assert np.array_equal(flags, g[key + "_flags"]), key
            within_a1(pairs, g[key + "_pairs"])
            cols = np.full((len(points), 16, 3), np.nan)
            operators.assemble_columns(g[key + "_pairs"], *layout, cols, device)
            assert np.array_equal(cols.view(np.uint64), g[key + "_columns"].view(np.uint64)), key
            fused, fflags = operators.ring_columns(points, wing["starts"], wing["directions"], wing["lengths"],
                                                   radius, model, mode == "raise", *layout, device)
            assert np.array_equal(fflags, g[key + "_flags"]), key
            scale = np.linalg.norm(g[key + "_pairs"], axis=-1).sum(axis=1)
            err = np.linalg.norm(fused - g[key + "_columns"], axis=-1)
            assert np.all(err <= 1e-12 * scale[:, None] + 1e-300), key


def test_ring_operator_of_a_64_panel_wing_and_lattice(device):
    """The 64-panel wing (the VSM Jacobian size) and the lattice wake as 1,024 x 4,207 pair matrix: GPU against the
    oracle's bit-exact restatement."""
    from openfawe_b200 import engine, operators, wakes
    wing = wakes.ring_wing()
    layout = (wing["column_ptr"], wing["column_segment"], wing["column_sign"])
    ref_pairs, ref_flags = O.pair_matrix(wing["points"], wing["starts"], wing["directions"], wing["lengths"],
                                         wing["radius"], 2, True)
    ref_cols = O.assemble_columns(ref_pairs, *layout)
    cols, flags = operators.ring_columns(wing["points"], wing["starts"], wing["directions"], wing["lengths"],
                                         wing["radius"], 2, True, *layout, device)
    assert not flags.any() and np.array_equal(flags, ref_flags)
    scale = np.linalg.norm(ref_pairs, axis=-1).sum(axis=1)
    assert np.all(np.linalg.norm(cols - ref_cols, axis=-1) <= 1e-12 * scale[:, None])
    case = wakes.lattice()
    src = engine.Sources(case["starts"], case["directions"], case["lengths"], case["gamma"], case["radius"], device)
    pairs, flags = operators.pair_matrix_device(case["points"], src, case["model"], True)
    ref, rflags = O.pair_matrix(case["points"], case["starts"], case["directions"], case["lengths"], case["radius"],
                                case["model"], True)
    assert np.array_equal(flags.cpu().numpy(), rflags)
    within_a1(pairs.cpu().numpy(), ref)
    # the Gamma-weighted row sums of the pair matrix are the direct sum
    u, _ = engine.direct(src, engine.Targets(case["points"], None, device), case["model"], "raise", "fp64")
    rows = (pairs * src.gamma[None, :, None]).sum(dim=1)
    np.testing.assert_allclose(rows.cpu().numpy(), u.cpu().numpy(), rtol=1e-10, atol=1e-12 * float(u.abs().max()))


def test_operator_argument_errors(device):
    from openfawe_b200 import operators, wakes
    wing = wakes.ring_wing(panels=4, rows=1)
    pairs = np.zeros((4, len(wing["starts"]), 3))
    out = np.zeros((4, 4, 3))
    with pytest.raises(ValueError):
        operators.assemble_columns(pairs, wing["column_ptr"], wing["column_segment"] + 1000, wing["column_sign"], out,
                                   device)
    with pytest.raises(ValueError):
        operators.assemble_columns(pairs, wing["column_ptr"][::-1], wing["column_segment"], wing["column_sign"], out,
                                   device)
