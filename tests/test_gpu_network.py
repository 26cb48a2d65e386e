"""Exclusion bookkeeping on the GPU (bs_incident_pairs, bs_exclusion_csr) against the reference's outputs and the
oracle.  Integer work: every comparison is exact (array_equal)."""
import numpy as np
import pytest

from conftest import golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_incident_pairs_and_csr_match_reference_fixtures(device):
    from openfawe_b200 import network
    g = golden("network.npz")
    for seed in (1, 2):
        nodes, edges, first = g[f"n{seed}_nodes"], g[f"n{seed}_edges"], int(g[f"n{seed}_first"])
        for f in (first, 0, len(nodes)):
            got = network.incident_pairs(nodes, edges, f, device)
            assert got.dtype == np.int64 and np.array_equal(got, g[f"n{seed}_f{f}_pairs"]), (seed, f)
    for name in "abcd":
        ptr, seg = network.exclusion_csr(int(g[f"x{name}_count"]), g[f"x{name}_pairs"], device)
        assert np.array_equal(ptr, g[f"x{name}_ptr"]) and np.array_equal(seg, g[f"x{name}_seg"]), name


def shed_network(rows, seed, duplicate=0.3):
    """A rotor-sheet wake whose shed nodes (after the first row) partly repeat earlier nodes' coordinates, as a
    wake step's convected nodes sit on the previous step's nodes."""
    from openfawe_b200 import wakes
    case = wakes.rotor_sheet(rows, seed=seed, targets=1)
    nodes, edges = case["nodes"].copy(), case["edges"]
    first = 219 if rows > 1 else 0
    rng = np.random.default_rng(seed)
    k = int(duplicate * (len(nodes) - first))
    dst = rng.choice(np.arange(first, len(nodes)), k, replace=False)
    nodes[dst] = nodes[rng.integers(0, len(nodes), k)]
    return nodes, edges, first


def test_incident_pairs_large_network_against_oracle(device):
    from openfawe_b200 import network
    for rows, seed in ((40, 1), (468, 2)):
        nodes, edges, first = shed_network(rows, seed)
        ref = O.incident_pairs(nodes, edges, first)
        got = network.incident_pairs(nodes, edges, first, device)
        assert len(ref) > len(edges) and np.array_equal(got, ref), rows
    # a capacity too small is reported, then the call with the right size gives the same pairs
    import torch
    nodes, edges, first = shed_network(40, 3)
    t = network.incident_pairs_device(torch.as_tensor(nodes, device=device), torch.as_tensor(edges, device=device),
                                      first, capacity=1)
    assert np.array_equal(t.cpu().numpy(), O.incident_pairs(nodes, edges, first))


def test_exclusion_csr_large_against_oracle(device):
    from openfawe_b200 import network
    rng = np.random.default_rng(7)
    n, m = 20570, 819890
    pairs = np.column_stack((rng.integers(0, n, 400_000), rng.integers(0, m, 400_000)))
    pairs = np.vstack([pairs, pairs[:50_000]])  # repeats
    ptr, seg = network.exclusion_csr(n, pairs, device)
    rp, rs = O.exclusion_csr(n, pairs)
    assert np.array_equal(ptr, rp) and np.array_equal(seg, rs)
    # the incident pairs of a wake feed the CSR exactly as the reference chains them (wake.py:428-431, vortex.py:470)
    nodes, edges, first = shed_network(120, 4)
    inc = network.incident_pairs(nodes, edges, first, device)
    ptr, seg = network.exclusion_csr(len(nodes) - first, inc, device)
    rp, rs = O.exclusion_csr(len(nodes) - first, O.incident_pairs(nodes, edges, first))
    assert np.array_equal(ptr, rp) and np.array_equal(seg, rs)


def test_network_errors(device):
    from openfawe_b200 import network
    nodes = np.zeros((4, 3))
    with pytest.raises(ValueError):
        network.incident_pairs(nodes, np.array([[0, 4]]), 0, device)
    with pytest.raises(ValueError):
        network.incident_pairs(nodes, np.array([[0, 1]]), 5, device)
    with pytest.raises(ValueError):
        network.exclusion_csr(3, np.array([[3, 0]]), device)
    with pytest.raises(ValueError):
        network.exclusion_csr(3, np.array([[-1, 0]]), device)
    assert network.incident_pairs(nodes, np.zeros((0, 2), dtype=np.int64), 0, device).shape == (0, 2)
    # all nodes equal: every end of every segment matches every free point
    got = network.incident_pairs(nodes, np.array([[0, 1], [2, 3]]), 1, device)
    assert np.array_equal(got, O.incident_pairs(nodes, np.array([[0, 1], [2, 3]]), 1))
