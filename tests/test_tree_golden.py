"""Bit-exact parity of the host tree (cdfmm.UniformTree) with the reference.

Golden vectors: the reference's own UniformTree (tests/golden/make_golden.py).
Pins upstream src/uniform_tree.cpp:129-523 semantics: root cube, leaf
assignment with the 1e-12 tolerance and clamping, stable Morton order,
half-open ranges with the population-size sentinel, list1/list2 order.
"""

import numpy as np
import pytest

import cdfmm
from conftest import GOLDEN, group_names, load_group


def build(g):
    o = cdfmm.UniformTreeOptions()
    o.max_level = int(g["depth"])
    if bool(g["has_root"]):
        r = g["root_in"]
        o.root_centre = cdfmm.Vec3(*r[:3])
        o.root_half_width = float(r[3])
    return cdfmm.UniformTree(g["sources"], g["targets"], o)


@pytest.mark.parametrize("name", group_names("trees.npz"))
def test_tree_permutations_and_ranges_bit_exact(name):
    g = load_group("trees.npz", name)
    t = build(g)
    np.testing.assert_array_equal(np.array(t.source_permutation), g["source_permutation"])
    np.testing.assert_array_equal(np.array(t.target_permutation), g["target_permutation"])
    ranges = np.array([(n.source_begin, n.source_end, n.target_begin, n.target_end) for n in t.nodes])
    np.testing.assert_array_equal(ranges, g["ranges"])
    assert (t.root_centre.x, t.root_centre.y, t.root_centre.z) == tuple(g["root_centre"])
    assert t.root_half_width == g["root_half_width"]


@pytest.mark.parametrize("depth", [2, 3])
def test_tree_lists_bit_exact(depth):
    data = np.load(f"{GOLDEN}/lists.npz")
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth
    t = cdfmm.UniformTree(np.array([[0.0, 0, 0], [1.0, 1, 1]]), o)
    l1 = [list(n.list1) for n in t.nodes]
    l2 = [list(n.list2) for n in t.nodes]
    np.testing.assert_array_equal(np.cumsum([0] + [len(v) for v in l1]), data[f"d{depth}__l1_off"])
    np.testing.assert_array_equal(np.array([i for v in l1 for i in v]), data[f"d{depth}__l1"])
    np.testing.assert_array_equal(np.cumsum([0] + [len(v) for v in l2]), data[f"d{depth}__l2_off"])
    np.testing.assert_array_equal(np.array([i for v in l2 for i in v]), data[f"d{depth}__l2"])


def test_node_counts_and_morton():
    # upstream tests/test_uniform_tree.cpp:11-28
    for depth, count in ((0, 1), (1, 9), (2, 73), (3, 585)):
        o = cdfmm.UniformTreeOptions()
        o.max_level = depth
        assert len(cdfmm.UniformTree(np.zeros((1, 3)), o).nodes) == count
    assert cdfmm.node_index(3, 5, 3, 7) == cdfmm.level_offset(3) + cdfmm.morton_encode(5, 3, 7)
    for xyz in ((0, 0, 0), (5, 3, 7), (1023, 17, 900)):
        assert tuple(cdfmm.morton_decode(cdfmm.morton_encode(*xyz))) == xyz


def test_tree_rejects_points_outside_explicit_root():
    o = cdfmm.UniformTreeOptions()
    o.max_level = 2
    o.root_centre = cdfmm.Vec3(0, 0, 0)
    o.root_half_width = 1.0
    with pytest.raises(ValueError, match="outside the requested root box"):
        cdfmm.UniformTree(np.array([[1.1, 0, 0]]), o)
    o.root_half_width = -1.0
    with pytest.raises(ValueError, match="root_half_width must be positive"):
        cdfmm.UniformTree(np.array([[0.1, 0, 0]]), o)
    o2 = cdfmm.UniformTreeOptions()
    o2.max_level = -1
    with pytest.raises(ValueError, match="max_level must be >= 0"):
        cdfmm.UniformTree(np.array([[0.1, 0, 0]]), o2)


def test_tree_large_uniform_matches_oracle():
    import oracle

    rng = np.random.default_rng(77)
    x = rng.uniform(0, 1, size=(200_000, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 5
    t = cdfmm.UniformTree(x, x, o)
    ref = oracle.tree(x, x, 5)
    np.testing.assert_array_equal(np.array(t.source_permutation), ref["source_permutation"])
    ranges = np.array([(n.source_begin, n.source_end, n.target_begin, n.target_end) for n in t.nodes])
    np.testing.assert_array_equal(ranges, ref["ranges"])
