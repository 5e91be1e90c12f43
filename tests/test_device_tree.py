"""Plans built from raw positions: the device octree and the operator cache.

cdfmm_b200_plan_create_from_points builds the uniform octree on the GPU.  Its
root cube, stable Morton ordering and leaf ranges must equal the reference's
UniformTree bit for bit (upstream src/uniform_tree.cpp:129-357): the GPU
tests check it against the golden trees generated by the reference itself
(tests/golden/trees.npz) and against cdfmm.UniformTree on larger and
degenerate inputs (leaf-boundary coordinates, duplicates, signed zeros,
explicit roots), and check that a plan built this way evaluates bit-identically
to the plan built from the host tree.  The CPU tests cover the argument
checks and the on-disk M2L operator cache (CDFMM_B200_OPERATOR_CACHE).
"""

import os
import subprocess
import sys

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
from conftest import group_names, load_group

PY = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dip-fmm_b200", "python")


def host_tree(src, tgt, depth, centre=None, half_width=None):
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth
    if centre is not None:
        o.root_centre = cdfmm.Vec3(*centre)
    if half_width is not None:
        o.root_half_width = float(half_width)
    return cdfmm.UniformTree(src, src if tgt is None else tgt, o)


def assert_same_tree(plan, t, src, tgt):
    d = plan.tree()
    rc = t.root_centre
    assert tuple(d["root_centre"]) == (rc.x, rc.y, rc.z)
    np.testing.assert_array_equal(np.signbit(d["root_centre"]), np.signbit([rc.x, rc.y, rc.z]))
    assert d["root_half_width"] == t.root_half_width
    np.testing.assert_array_equal(d["source_permutation"], np.array(t.source_permutation))
    np.testing.assert_array_equal(d["target_permutation"], np.array(t.target_permutation))
    np.testing.assert_array_equal(d["leaf_source_offsets"], np.asarray(t.leaf_source_offsets()))
    np.testing.assert_array_equal(d["leaf_target_offsets"], np.asarray(t.leaf_target_offsets()))
    np.testing.assert_array_equal(d["sorted_source_positions"], np.asarray(src)[d["source_permutation"]])
    tg = src if tgt is None else tgt
    np.testing.assert_array_equal(d["sorted_target_positions"], np.asarray(tg)[d["target_permutation"]])


# ---------------------------------------------------------------- CPU -------

def test_points_plan_argument_checks():
    x = np.random.default_rng(0).random((10, 3))
    with pytest.raises(ValueError, match="self_map needs targets"):
        cdfmm_b200.DevicePlan.from_points(x, 3, 2, targets=x, self_map=True)
    with pytest.raises(ValueError, match="root_half_width must be positive"):
        cdfmm_b200.DevicePlan.from_points(x, 3, 2, root_half_width=-1.0)
    with pytest.raises(ValueError, match="depth must be in"):
        cdfmm_b200.DevicePlan.from_points(x, 3, 9)


def test_m2l_stencil_matches_the_matrix_generator():
    T, _ = cdfmm_b200.m2l_stencil(4)
    n = 35
    assert T.shape == (343, n, n)
    for t in [(2, 0, 0), (-3, 1, 2), (3, 3, -3), (0, -2, 1)]:
        slot = (t[0] + 3) * 49 + (t[1] + 3) * 7 + (t[2] + 3)
        np.testing.assert_array_equal(T[slot], cdfmm_b200.m2l_matrix(4, np.array(t, float)).T)
    near = [(a + 3) * 49 + (b + 3) * 7 + (c + 3) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    assert not T[near].any()
    _, src = cdfmm_b200.m2l_stencil(4)
    assert src == cdfmm_b200.STENCIL_PROCESS


def _stencil_in_child(cache_dir, order):
    code = (f"import sys; sys.path.insert(0, {PY!r}); import numpy as np, cdfmm_b200; "
            f"T, s = cdfmm_b200.m2l_stencil({order}); np.save({os.path.join(str(cache_dir), 'out.npy')!r}, T); "
            "print(s)")
    env = dict(os.environ, CDFMM_B200_OPERATOR_CACHE=str(cache_dir))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return int(r.stdout.strip()), np.load(os.path.join(str(cache_dir), "out.npy"))


def test_operator_cache_on_disk(tmp_path):
    order = 5
    src0, T0 = _stencil_in_child(tmp_path, order)
    path = tmp_path / f"m2l_p{order}.bin"
    assert src0 == cdfmm_b200.STENCIL_COMPUTED and path.exists()
    src1, T1 = _stencil_in_child(tmp_path, order)
    assert src1 == cdfmm_b200.STENCIL_DISK
    np.testing.assert_array_equal(T0, T1)
    # a damaged file fails its checksum: recomputed and rewritten
    raw = bytearray(path.read_bytes())
    raw[len(raw) // 2] ^= 0x40
    path.write_bytes(bytes(raw))
    src2, T2 = _stencil_in_child(tmp_path, order)
    assert src2 == cdfmm_b200.STENCIL_COMPUTED
    np.testing.assert_array_equal(T0, T2)
    src3, _ = _stencil_in_child(tmp_path, order)
    assert src3 == cdfmm_b200.STENCIL_DISK
    # a truncated file is ignored too
    path.write_bytes(path.read_bytes()[:1000])
    src4, T4 = _stencil_in_child(tmp_path, order)
    assert src4 == cdfmm_b200.STENCIL_COMPUTED
    np.testing.assert_array_equal(T0, T4)
    assert not [p for p in os.listdir(tmp_path) if ".tmp." in p]


# ---------------------------------------------------------------- GPU -------

@pytest.mark.gpu
@pytest.mark.parametrize("name", group_names("trees.npz"))
def test_device_tree_matches_reference_golden_trees(name):
    g = load_group("trees.npz", name)
    depth = int(g["depth"])
    kw = {}
    if bool(g["has_root"]):
        r = g["root_in"]
        kw = {"root_centre": r[:3], "root_half_width": float(r[3])}
    plan = cdfmm_b200.DevicePlan.from_points(g["sources"], 2, depth, targets=g["targets"], **kw)
    d = plan.tree()
    np.testing.assert_array_equal(d["source_permutation"], g["source_permutation"])
    np.testing.assert_array_equal(d["target_permutation"], g["target_permutation"])
    assert tuple(d["root_centre"]) == tuple(g["root_centre"])
    assert d["root_half_width"] == g["root_half_width"]
    # leaf ranges against the reference's node ranges (leaf level, non-empty)
    ranges = g["ranges"]
    base = ((1 << (3 * depth)) - 1) // 7
    so, to = d["leaf_source_offsets"], d["leaf_target_offsets"]
    for m in range(1 << (3 * depth)):
        sb, se, tb, te = ranges[base + m]
        if so[m + 1] > so[m]:
            assert (sb, se) == (so[m], so[m + 1])
        if to[m + 1] > to[m]:
            assert (tb, te) == (to[m], to[m + 1])
    plan.close()


def _cases():
    rng = np.random.default_rng(2024)
    u = rng.random((20000, 3))
    # coordinates on leaf boundaries of the depth-3 grid of [0, 1]^3, repeats
    g = rng.integers(0, 9, size=(5000, 3)) / 8.0
    g[:8] = [[0, 0, 0], [1, 1, 1], [0, 1, 0], [1, 0, 1], [0.5, 0.5, 0.5], [0.125, 0.875, 0.25], [1, 1, 1], [0, 0, 0]]
    # signed zeros on the box faces
    z = rng.uniform(-1, 1, size=(3000, 3))
    z[::7, 0] = -0.0
    z[3::7, 0] = 0.0
    z[::5, 1] = 0.0
    z[[0, 1], 2] = [0.0, -0.0]
    # a plane of signed zeros (x), a face of them (y >= 0): the root centre
    # takes the sign of the first zero, as the host tree's min / max do
    p = rng.random((2000, 3))
    p[:, 0] = np.where(rng.random(2000) < 0.5, -0.0, 0.0)
    p[0, 0] = -0.0
    p[::3, 1] = -0.0
    c = np.concatenate([rng.normal(0.3, 0.01, size=(6000, 3)), rng.normal(0.7, 0.2, size=(2000, 3))])
    return {"uniform": (u, None), "grid": (g, None), "signed_zero_faces": (z, None), "zero_plane": (p, None),
            "clustered_two_pop": (c, rng.random((7000, 3)) * 2 - 0.5)}


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(_cases().keys()))
@pytest.mark.parametrize("depth", [0, 1, 3, 5])
def test_device_tree_matches_host_tree(case, depth):
    src, tgt = _cases()[case]
    plan = cdfmm_b200.DevicePlan.from_points(src, 3, depth, targets=tgt)
    assert_same_tree(plan, host_tree(src, tgt, depth), src, tgt)
    plan.close()


@pytest.mark.gpu
def test_device_tree_explicit_roots_and_errors():
    rng = np.random.default_rng(7)
    x = rng.random((4000, 3))
    for centre, hw in [((0.5, 0.5, 0.5), 0.5), ((0.5, 0.5, 0.5), None), (None, 0.75), ((0.0, 0.0, 0.0), 1.0 + 1e-13)]:
        plan = cdfmm_b200.DevicePlan.from_points(x, 3, 4, root_centre=centre, root_half_width=hw)
        assert_same_tree(plan, host_tree(x, None, 4, centre, hw), x, None)
        plan.close()
    # a point just inside the 1e-12 tolerance is kept, one beyond it is refused
    y = x.copy()
    y[17] = (1.0 + 0.5e-12, 0.5, 0.5)
    plan = cdfmm_b200.DevicePlan.from_points(y, 3, 4, root_centre=(0.5, 0.5, 0.5), root_half_width=0.5)
    assert_same_tree(plan, host_tree(y, None, 4, (0.5, 0.5, 0.5), 0.5), y, None)
    plan.close()
    y[17] = (1.0 + 1e-9, 0.5, 0.5)
    with pytest.raises(ValueError, match="outside the requested root box"):
        cdfmm_b200.DevicePlan.from_points(y, 3, 4, root_centre=(0.5, 0.5, 0.5), root_half_width=0.5)
    y[17] = (np.nan, 0.5, 0.5)
    with pytest.raises(ValueError, match="outside the requested root box"):
        cdfmm_b200.DevicePlan.from_points(y, 3, 4)
    # coincident points span no volume: an explicit half width is needed
    one = np.array([[0.25, -1.0, 3.0], [0.25, -1.0, 3.0]])
    with pytest.raises(ValueError, match="span no volume"):
        cdfmm_b200.DevicePlan.from_points(one, 3, 2)
    plan = cdfmm_b200.DevicePlan.from_points(one, 3, 2, root_half_width=0.5)
    assert_same_tree(plan, host_tree(one, None, 2, None, 0.5), one, None)
    plan.close()
    # targets outside an explicit root
    with pytest.raises(ValueError, match="outside the requested root box"):
        cdfmm_b200.DevicePlan.from_points(x, 3, 4, targets=x + 2.0, root_centre=(0.5, 0.5, 0.5), root_half_width=0.5)


@pytest.mark.gpu
def test_device_tree_from_device_positions():
    import torch

    rng = np.random.default_rng(11)
    x = rng.normal(size=(30000, 3))
    y = rng.random((5000, 3))
    a = cdfmm_b200.DevicePlan.from_points(torch.from_numpy(x).cuda(), 4, 4, targets=torch.from_numpy(y).cuda())
    assert_same_tree(a, host_tree(x, y, 4), x, y)
    a.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order,depth,K", [(6, 4, 1), (6, 4, 8), (8, 3, 4)])
def test_points_plan_evaluates_like_the_host_tree_plan(order, depth, K):
    rng = np.random.default_rng(100 + K)
    n = 50000
    x = np.concatenate([rng.random((n - 5000, 3)), rng.normal(0.4, 0.02, size=(5000, 3))])
    m = rng.normal(size=(K, n, 3))
    t = host_tree(x, None, depth)
    ref = cdfmm_b200.DevicePlan.from_tree(t, order, max_states=K)
    ref.set_self_indices(np.array(t.source_inverse_permutation)[np.array(t.target_permutation)])
    dev = cdfmm_b200.DevicePlan.from_points(x, order, depth, max_states=K)
    for plan in (ref, dev):
        # one pinned M2L shape: the autotuner's choice may differ between plans
        shapes = plan.m2l_shapes()
        if shapes:
            plan.set_m2l_shape(*shapes[0])
    a = ref.evaluate(m, output="both")
    b = dev.evaluate(m, output="both")
    np.testing.assert_array_equal(a["H"], b["H"])
    np.testing.assert_array_equal(a["phi"], b["phi"])
    sa, sb = ref.stats(), dev.stats()
    for key in ("p2p_pairs", "m2l_interactions", "m2l_classes"):
        assert sa[key] == sb[key]
    ref.close()
    dev.close()
