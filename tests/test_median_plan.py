"""The premise of the planned median build (csrc/bs_tree_build.cu build_median), on the CPU against the oracle.

The reference's median split (vortex_tree.build_tree, restated in oracle/) splits a node larger than a leaf at the
middle of its range unless its midpoints' box has no extent, so without such a node the topology (ranges and children
in depth-first numbering) follows from the segment count and the leaf size alone; the device build queues every level
on that plan and only reads back whether a degenerate node occurred.  Checked here for random midpoints at many sizes
and leaf sizes, and for a cluster of coincident midpoints, which the plan must not claim to match.
"""
import numpy as np

from oracle import oracle as O


def planned_topology(m, leaf):
    """(lo, hi, left, right) of the all-split plan: level by level in order (as the build numbers nodes), then
    renumbered depth first (left child, then right) as the reference numbers them."""
    lo, hi, left, right = [0], [m], [-1], [-1]
    level = [0]
    while level:
        following = []
        for node in level:
            a, b = lo[node], hi[node]
            if b - a > leaf:
                middle = (a + b) // 2
                f = len(lo)
                lo += [a, middle]
                hi += [middle, b]
                left += [-1, -1]
                right += [-1, -1]
                left[node], right[node] = f, f + 1
                following += [f, f + 1]
        level = following
    count = len(lo)
    number = [0] * count
    olo, ohi, oleft, oright = [0] * count, [0] * count, [-1] * count, [-1] * count
    olo[0], ohi[0] = lo[0], hi[0]
    assigned, stack = 1, [0]
    while stack:
        node = stack.pop()
        if left[node] < 0:
            continue
        f, g = assigned, assigned + 1
        assigned += 2
        number[left[node]], number[right[node]] = f, g
        oleft[number[node]], oright[number[node]] = f, g
        olo[f], ohi[f] = lo[left[node]], hi[left[node]]
        olo[g], ohi[g] = lo[right[node]], hi[right[node]]
        stack += [right[node], left[node]]
    return np.array(olo), np.array(ohi), np.array(oleft), np.array(oright)


def test_median_topology_follows_from_count_and_leaf():
    rng = np.random.default_rng(8)
    for m, leaf in ((1, 1), (7, 8), (9, 8), (100, 1), (257, 4), (1000, 32), (3001, 7), (5000, 16)):
        mid = rng.normal(size=(m, 3)) * [20.0, 5.0, 2.0]
        ref = O.build_tree(mid, leaf)
        for got, want, name in zip(planned_topology(m, leaf), ref[1:5], ("lo", "hi", "left", "right")):
            assert np.array_equal(got, want), (m, leaf, name)


def test_a_node_without_extent_departs_from_the_plan():
    rng = np.random.default_rng(9)
    mid = np.concatenate((rng.normal(size=(600, 3)), np.full((40, 3), 5.0)))
    ref = O.build_tree(mid, 4)
    planned = planned_topology(len(mid), 4)
    assert len(planned[0]) != ref[5] or not all(np.array_equal(a, b) for a, b in zip(planned, ref[1:5]))
