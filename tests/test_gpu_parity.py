"""GPU parity tests of the B200 path (run with -m gpu on a B200).

Checked against (a) golden vectors of the upstream reference's CpuStatic
FP32 / FP64 backends and FP64 direct sum (tests/golden/fmm.npz), (b) the CPU
oracle (oracle/, FP64 restatement pinned to the same goldens), and (c) the
device FP64 direct sum.  Tolerances are the reference's own FP32 bars:
rel-L2(H) <= 3e-5 FP32 vs FP64 (upstream tests/test_precision.cpp:332-367),
per-element rtol 2e-5 (python_tests/test_fmm_precision.py:56-74).
"""

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
import oracle
from conftest import group_names, load_group

pytestmark = pytest.mark.gpu

FP32_REL_L2 = 3e-5


def make_fmm(g_or_src, tgt=None, order=4, depth=3, root=None, fixed=None, max_states=1, m2l=None):
    o = cdfmm.UniformFmmOptions()
    o.expansion_order = order
    o.tree.max_level = depth
    o.max_states = max_states
    if m2l is not None:
        o.b200_m2l = m2l
    if root is not None:
        o.tree.root_centre = cdfmm.Vec3(*root[:3])
        o.tree.root_half_width = float(root[3])
    if fixed is not None:
        o.fixed_target_source_indices = list(map(int, fixed))
    return cdfmm.UniformFmm(g_or_src, tgt, o)


def golden_fmm(name):
    g = load_group("fmm.npz", name)
    root = g["root_in"] if bool(g["has_root"]) else None
    f = make_fmm(g["sources"], g["targets"], int(g["order"]), int(g["depth"]), root)
    ids = g["identities"] if g["identities"].size else None
    return g, f, ids


@pytest.mark.parametrize("name", group_names("fmm.npz"))
def test_evaluate_matches_reference_cpustatic(name):
    g, f, ids = golden_fmm(name)
    r = f.evaluate(g["moments"], output="both", target_source_indices=None if ids is None else ids.tolist())
    assert r["H"].dtype == np.float32 and r["phi"].dtype == np.float32
    assert oracle.rel_l2(r["H"], g["H64"]) < FP32_REL_L2
    assert oracle.rel_l2(r["H"], g["H32"]) < FP32_REL_L2
    assert oracle.rel_l2(r["phi"], g["phi64"]) < FP32_REL_L2
    assert f.static_plan_statistics["transfer_classes"] == int(g["transfer_classes"])
    assert f.static_plan_statistics["interactions"] == int(g["interactions"])
    if int(g["depth"]) == 0:
        assert oracle.rel_l2(r["H"], g["H_direct"]) < 5e-6


@pytest.mark.parametrize("m2l,bar", [("FLOAT32", 2e-5), ("SPLIT_BF16", 1e-4)])
def test_stage_expansions_match_reference(m2l, bar):
    """Per-node multipoles and locals against the reference's FP32 plan.  With
    the FP32 SIMT M2L every stage is FP32 like the reference's (bar 2e-5 of
    each node's largest coefficient); with the split-BF16 M2L each operand
    carries ~2^-17 relative error (hi + lo in 16 mantissa bits, lo x lo
    dropped), which sums over a node's ~6,600 terms to a few 1e-5 of its
    locals (bar 1e-4)."""
    g = load_group("fmm.npz", "expansions_p4_d3")
    f = make_fmm(g["sources"], g["targets"], int(g["order"]), int(g["depth"]),
                 m2l=getattr(cdfmm.B200M2L, m2l))
    ids = g["identities"]
    f.evaluate(g["moments"], target_source_indices=ids.tolist())
    nn = len(f.tree.nodes)
    M = np.stack([f.multipole(i) for i in range(nn)]).astype(np.float64)
    L = np.stack([f.local(i) for i in range(nn)]).astype(np.float64)
    for what, ours, ref in (("M", M, g["M32"].astype(np.float64)), ("L", L, g["L32"].astype(np.float64))):
        scale = np.abs(ref).max(axis=1)
        err = np.abs(ours - ref).max(axis=1)
        bad = np.nonzero(err > bar * scale)[0]
        detail = [(int(i), f.tree.nodes[int(i)].level, float(err[i]), float(scale[i]),
                   float(np.abs(ours[i]).max())) for i in bad[:5]]
        assert bad.size == 0, f"{what}: {bad.size} nodes differ, first (node, level, err, ref max, ours max): {detail}"


def test_field_only_and_potential_only_outputs():
    g, f, ids = golden_fmm("small_p4_d3")
    both = f.evaluate(g["moments"], output="both", target_source_indices=ids.tolist())
    field = f.evaluate(g["moments"], output="field", target_source_indices=ids.tolist())
    pot = f.evaluate(g["moments"], output="potential", target_source_indices=ids.tolist())
    np.testing.assert_array_equal(field["H"], both["H"])
    np.testing.assert_array_equal(field["phi"], 0.0)
    np.testing.assert_array_equal(pot["phi"], both["phi"])
    np.testing.assert_array_equal(pot["H"], 0.0)


def test_repeated_state_and_zero_moments_reset():
    g, f, ids = golden_fmm("small_p2_d2")
    a = f.evaluate(g["moments"], target_source_indices=ids.tolist())["H"]
    z = f.evaluate(np.zeros_like(g["moments"]), target_source_indices=ids.tolist())["H"]
    b = f.evaluate(g["moments"], target_source_indices=ids.tolist())["H"]
    np.testing.assert_array_equal(z, 0.0)
    np.testing.assert_array_equal(a, b)
    for node in f.tree.nodes:
        assert np.all(np.isfinite(f.local(node.index)))


def test_user_order_is_preserved_under_permutation():
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (500, 3))
    m = rng.normal(size=(500, 3))
    perm = rng.permutation(500)
    f1 = make_fmm(x, x, 4, 3)
    f2 = make_fmm(x[perm], x[perm], 4, 3)
    h1 = f1.evaluate(m, target_source_indices=list(range(500)))["H"]
    h2 = f2.evaluate(m[perm], target_source_indices=list(range(500)))["H"]
    np.testing.assert_allclose(h2, h1[perm], rtol=2e-5, atol=2e-5 * np.abs(h1).max())


def test_identity_map_contract():
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, (300, 3))
    m = rng.normal(size=(300, 3))
    ids = np.arange(300)
    f = make_fmm(x, x, 4, 2, fixed=ids)
    implicit = f.evaluate(m)["H"]
    explicit = f.evaluate(m, target_source_indices=ids.tolist())["H"]
    np.testing.assert_array_equal(implicit, explicit)
    changed = ids.copy()
    changed[0] = 5
    with pytest.raises(ValueError, match="identity map changed"):
        f.evaluate(m, target_source_indices=changed.tolist())
    with pytest.raises(ValueError, match="incorrect length"):
        make_fmm(x, x, 4, 2).evaluate(m, target_source_indices=[0, 1])
    with pytest.raises(ValueError, match="invalid index"):
        make_fmm(x, x, 4, 2).evaluate(m, target_source_indices=[300] * 300)
    with pytest.raises(ValueError, match="one dipole moment per source"):
        f.evaluate(m[:-1])


def test_coincident_non_self_pair_is_nan_like_reference():
    x = np.array([[0.1, 0.2, 0.3], [0.1, 0.2, 0.3], [0.7, 0.6, 0.5], [0.4, 0.9, 0.2]])
    m = np.ones((4, 3))
    f = make_fmm(x, x, 3, 1)
    with_ids = f.evaluate(m, target_source_indices=[0, 1, 2, 3])["H"]
    assert np.isnan(with_ids[0]).all() and np.isnan(with_ids[1]).all()
    assert np.isfinite(with_ids[2:]).all()


def test_empty_geometry_is_accepted():
    o = cdfmm.UniformFmmOptions()
    o.tree.max_level = 2
    f = cdfmm.UniformFmm(np.zeros((0, 3)), np.zeros((0, 3)), o)
    r = f.evaluate(np.zeros((0, 3)))
    assert r["H"].shape == (0, 3)
    f2 = cdfmm.UniformFmm(np.random.default_rng(0).uniform(0, 1, (20, 3)), np.zeros((0, 3)), o)
    assert f2.evaluate(np.ones((20, 3)))["H"].shape == (0, 3)


def test_upward_pass_root_matches_oracle():
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (400, 3))
    m = rng.normal(size=(400, 3))
    o = cdfmm.UniformFmmOptions()
    o.expansion_order = 5
    o.tree.max_level = 3
    o.tree.root_centre = cdfmm.Vec3(0, 0, 0)
    o.tree.root_half_width = 1.0
    f = cdfmm.UniformFmm(x, o)
    f.upward_pass(m)
    r = oracle.fmm(x, np.zeros((0, 3)), m, 5, 3, root_centre=[0, 0, 0], root_half_width=1.0, expansions=True)
    deg = oracle.basis(5).sum(axis=1)
    root_ref = r["M"][0] * 2.0 ** (-(deg + 2.0))
    np.testing.assert_allclose(f.root_multipole, root_ref, rtol=1e-5, atol=1e-5 * np.abs(root_ref).max())


@pytest.mark.parametrize("K", [2, 5, 8, 13, 16, 64])
def test_batched_states_match_single_state_calls(K):
    """K states in one call equal K single-state calls.  K >= 8 takes the
    split-BF16 tensor-core M2L (three products), so the bar there is the
    FP32 bar against FP64 rather than near bit-equality with the FP32 path."""
    rng = np.random.default_rng(100 + K)
    x = rng.uniform(0, 1, (3000, 3))
    ms = rng.normal(size=(K, 3000, 3)).astype(np.float32)
    f = make_fmm(x, x, 5, 3, max_states=K)
    ids = list(range(3000))
    batch = f.evaluate_states(ms, output="both", target_source_indices=ids)
    tol = 2e-6 if K < 8 else 2e-5
    for k in sorted({0, K // 2, K - 1}):
        single = f.evaluate(ms[k].astype(np.float64), output="both", target_source_indices=ids)
        assert oracle.rel_l2(batch["H"][k], single["H"]) < tol
        assert oracle.rel_l2(batch["phi"][k], single["phi"]) < tol
        ref = oracle.fmm(x, x, ms[k], 5, 3, identities=np.arange(3000))
        assert oracle.rel_l2(batch["H"][k], ref["H"]) < FP32_REL_L2
        assert oracle.rel_l2(batch["phi"][k], ref["phi"]) < FP32_REL_L2


@pytest.mark.parametrize("name", ["c0", "small_p6_d4", "p6_d4_explicit_root", "targets_partial_ids"])
def test_split_bf16_tensor_core_m2l_matches_reference(name):
    """The tcgen05 split-BF16 M2L forced on single-state golden cases."""
    g = load_group("fmm.npz", name)
    root = g["root_in"] if bool(g["has_root"]) else None
    f = make_fmm(g["sources"], g["targets"], int(g["order"]), int(g["depth"]), root, m2l=cdfmm.B200M2L.SPLIT_BF16)
    ids = g["identities"] if g["identities"].size else None
    r = f.evaluate(g["moments"], output="both", target_source_indices=None if ids is None else ids.tolist())
    assert f.cuda_plan_statistics["m2l_unique_matrix_count"] == int(g["transfer_classes"])
    assert oracle.rel_l2(r["H"], g["H64"]) < FP32_REL_L2
    assert oracle.rel_l2(r["phi"], g["phi64"]) < FP32_REL_L2
    assert oracle.rel_l2(r["H"], g["H32"]) < FP32_REL_L2


def test_c_abi_layouts_dtypes_and_transfer_counts():
    rng = np.random.default_rng(12)
    x = rng.uniform(0, 1, (2000, 3))
    t = rng.uniform(0.2, 0.8, (1000, 3))
    m = rng.normal(size=(3, 2000, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, t, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=3)
    sep = plan.evaluate(m, output="both")
    inter = plan.evaluate(m.astype(np.float32), output="both", layout=cdfmm_b200.LAYOUT_INTERLEAVED)
    np.testing.assert_allclose(inter["H"][..., 1:], sep["H"], rtol=1e-5, atol=1e-5 * np.abs(sep["H"]).max())
    np.testing.assert_allclose(inter["H"][..., 0], sep["phi"], rtol=1e-5, atol=1e-5 * np.abs(sep["phi"]).max())
    ref = oracle.fmm(x, t, m[1], 4, 3)
    assert oracle.rel_l2(sep["H"][1], ref["H"]) < FP32_REL_L2
    assert oracle.rel_l2(sep["phi"][1], ref["phi"]) < FP32_REL_L2
    st = plan.stats()
    assert st["evaluations"] == 2
    assert st["evaluation_h2d_bytes"] == 3 * 2000 * 3 * 8 + 3 * 2000 * 3 * 4
    assert st["evaluation_d2h_bytes"] == 3 * 1000 * 4 * 4 + 3 * 1000 * 4 * 4


def test_device_resident_arrays_through_c_abi():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(13)
    x = rng.uniform(0, 1, (4000, 3))
    m = rng.normal(size=(4, 4000, 3)).astype(np.float32)
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 5, max_states=4)
    host = plan.evaluate(m, output="both")
    dm = torch.from_numpy(m).cuda()
    dH = torch.zeros((4, 4000, 3), dtype=torch.float32, device="cuda")
    dphi = torch.zeros((4, 4000), dtype=torch.float32, device="cuda")
    plan.evaluate(dm, output="both", field=dH, potential=dphi)
    np.testing.assert_array_equal(dH.cpu().numpy(), host["H"])
    np.testing.assert_array_equal(dphi.cpu().numpy(), host["phi"])


def test_device_direct_fp64_matches_oracle():
    rng = np.random.default_rng(14)
    x = rng.uniform(0, 1, (1500, 3))
    m = rng.normal(size=(1500, 3))
    ids = np.arange(1500)
    phi_d, H_d = cdfmm_b200.direct_fp64(x, m, x, ids)
    phi_o, H_o = oracle.direct(x, m, x, ids)
    np.testing.assert_allclose(H_d, H_o, rtol=1e-11, atol=1e-11 * np.abs(H_o).max())
    np.testing.assert_allclose(phi_d, phi_o, rtol=1e-11, atol=1e-11 * np.abs(phi_o).max())


def test_large_uniform_accuracy_linearity_and_oracle():
    """N = 131072 at p = 6, d = 4 (~32 per leaf): accuracy vs the FP64 direct
    sum on a subsample, and linearity in the moments."""
    rng = np.random.default_rng(15)
    N = 131072
    x = rng.uniform(0, 1, (N, 3))
    d = rng.normal(size=(N, 3))
    m1 = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.uniform(0.5, 1.5, (N, 1))
    m2 = rng.normal(size=(N, 3))
    f = make_fmm(x, x, 6, 4, max_states=2)
    ids = np.arange(N)
    r1 = f.evaluate(m1, output="both", target_source_indices=ids.tolist())
    sub = rng.choice(N, 4096, replace=False)
    phi_ref, H_ref = cdfmm_b200.direct_fp64(x, m1, x[sub], sub)
    # p = 6 truncation error of the algorithm itself (the reference's FP32 and
    # an FP64 FMM show the same): ~3e-5 for H, ~2.6e-4 for phi at ~32 per leaf.
    assert oracle.rel_l2(r1["H"][sub], H_ref) < 5e-5
    assert oracle.rel_l2(r1["phi"][sub], phi_ref) < 5e-4
    both = f.evaluate_states(np.stack([m1, m2]).astype(np.float32), output="field",
                             target_source_indices=ids.tolist())["H"]
    comb = f.evaluate((2.0 * m1 - 0.5 * m2), output="field", target_source_indices=ids.tolist())["H"]
    assert oracle.rel_l2(comb, 2.0 * both[0] - 0.5 * both[1]) < 1e-5


def test_host_io_chunk_pipeline_matches_device_path():
    # Host-memory calls with >= 128 states run as a pipeline of 64-state
    # chunks (copies overlapping the evaluation); results must equal the
    # device path.
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(31)
    n, K = 4096, 130
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    host = plan.evaluate(m, output="both")
    st = plan.stats()
    assert st["evaluation_h2d_bytes"] == K * n * 3 * 4
    assert st["evaluation_d2h_bytes"] == K * n * 4 * 4
    dH = torch.zeros((K, n, 3), device="cuda")
    dphi = torch.zeros((K, n), device="cuda")
    plan.evaluate(torch.from_numpy(m).cuda(), output="both", field=dH, potential=dphi)
    torch.cuda.synchronize()
    # (the 130-state device call runs the FP32 SIMT M2L, the 64-state chunks
    # the split-BF16 tensor cores: equal to the split's rounding)
    assert oracle.rel_l2(host["H"], dH.cpu().numpy()) < 1e-5
    assert oracle.rel_l2(host["phi"], dphi.cpu().numpy()) < 1e-5
    for k in (37, 129):
        ref = oracle.fmm(x, x, m[k].astype(np.float64), 4, 3, identities=np.arange(n))
        assert oracle.rel_l2(host["H"][k], ref["H"]) < FP32_REL_L2
    plan.close()


@pytest.mark.parametrize("K,dtype,output", [(33, np.float32, "both"), (64, np.float32, "both"),
                                             (48, np.float64, "field"), (40, np.float32, "potential")])
def test_host_io_state_parts_match_device_path(K, dtype, output):
    # Host-memory calls with 32 <= K < 128 states run as one evaluation whose
    # copies overlap it in parts of about a quarter of the states (a multiple
    # of 8; the first part half as long); results must equal the
    # device-resident call's.
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(53 + K)
    n = 5000
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, n, 3)).astype(dtype)
    before = plan.stats()
    host = plan.evaluate(m, output=output)
    st = plan.stats()
    part = ((K + 3) // 4 + 7) // 8 * 8
    first = min(K, (part // 2 + 7) // 8 * 8)      # the first part is half as long
    n_parts = 1 + -(-(K - first) // part)
    assert st["evaluation_h2d_calls"] - before["evaluation_h2d_calls"] == n_parts
    assert st["evaluation_h2d_bytes"] - before["evaluation_h2d_bytes"] == K * n * 3 * np.dtype(dtype).itemsize
    per_target = {"both": 4, "field": 3, "potential": 1}[output]
    assert st["evaluation_d2h_bytes"] - before["evaluation_d2h_bytes"] == K * n * per_target * 4
    dH = torch.zeros((K, n, 3), device="cuda")
    dphi = torch.zeros((K, n), device="cuda")
    plan.evaluate(torch.from_numpy(m).cuda(), output=output, field=dH, potential=dphi)
    torch.cuda.synchronize()
    if output != "potential":
        assert oracle.rel_l2(host["H"], dH.cpu().numpy()) < 1e-6
    if output != "field":
        assert oracle.rel_l2(host["phi"], dphi.cpu().numpy()) < 1e-6
    for k in (0, K - 1):
        ref = oracle.fmm(x, x, m[k].astype(np.float64), 4, 3, identities=np.arange(n))
        if output != "potential":
            assert oracle.rel_l2(host["H"][k], ref["H"]) < FP32_REL_L2
        else:
            assert oracle.rel_l2(host["phi"][k], ref["phi"]) < FP32_REL_L2
    plan.close()


@pytest.mark.parametrize("output", ["both", "potential", "field"])
def test_host_io_state_parts_interleaved_layout(output):
    # The same pipeline writing (phi, Hx, Hy, Hz) per target: the later
    # parts add their near field onto the far field of one L2P; components
    # that were not requested stay 0 as in the device-resident call.
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(91)
    n, K = 4000, 64
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    host = plan.evaluate(m, output=output, layout=cdfmm_b200.LAYOUT_INTERLEAVED)["H"]
    dF = torch.zeros((K, n, 4), device="cuda")
    plan.evaluate(torch.from_numpy(m).cuda(), output=output, layout=cdfmm_b200.LAYOUT_INTERLEAVED, field=dF)
    torch.cuda.synchronize()
    dev = dF.cpu().numpy()
    assert host.shape == (K, n, 4)
    for c in range(4):
        wanted = (c == 0 and output != "field") or (c > 0 and output != "potential")
        if wanted:
            assert oracle.rel_l2(host[..., c], dev[..., c]) < 1e-6
        else:
            np.testing.assert_array_equal(host[..., c], 0.0)
            np.testing.assert_array_equal(dev[..., c], 0.0)
    plan.close()


def test_python_uniform_fmm_zero_copy_device_io():
    # cdfmm.UniformFmm.evaluate_into takes CUDA arrays (torch tensors) in user
    # order and writes the results in place: no host copies.
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(41)
    n, K = 3000, 4
    x = rng.uniform(0, 1, (n, 3))
    f = make_fmm(x, x, 4, 3, max_states=K)
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    ref = f.evaluate_states(m, output="both", target_source_indices=list(range(n)))
    dm = torch.from_numpy(m).cuda()
    dH = torch.zeros((K, n, 3), device="cuda")
    dphi = torch.zeros((K, n), device="cuda")
    f.evaluate_into(dm, dH, dphi, output="both")
    torch.cuda.synchronize()
    np.testing.assert_allclose(dH.cpu().numpy(), ref["H"], rtol=1e-6, atol=1e-6 * np.abs(ref["H"]).max())
    np.testing.assert_allclose(dphi.cpu().numpy(), ref["phi"], rtol=1e-6, atol=1e-6 * np.abs(ref["phi"]).max())
    with pytest.raises(ValueError, match="wrong shape"):
        f.evaluate_into(dm, dH[:, :10], dphi, output="both")
    with pytest.raises(ValueError, match="float32"):
        f.evaluate_into(dm.double(), dH, dphi, output="both")


@pytest.mark.parametrize("order,K", [(5, 16), (6, 64)])
def test_every_m2l_pipeline_shape_gives_the_same_field(order, K):
    # Each tensor-core M2L pipeline shape the autotuner may pick, pinned in
    # turn: shapes with the same hi/lo fusion are bit-identical, fused and
    # unfused agree to FP32 rounding, and all meet the FP32 bar against the
    # FP64 oracle FMM.
    rng = np.random.default_rng(71 + order)
    n = 6000
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, order, max_states=K, m2l_mode=cdfmm_b200.M2L_BF16X3)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    shapes = plan.m2l_shapes()
    assert len(shapes) >= 2 and any(f for _, _, f in shapes) and any(not f for _, _, f in shapes)
    results = {}
    for mt, st, fused in shapes:
        plan.set_m2l_shape(mt, st, fused)
        H = plan.evaluate(m, output="field")["H"].copy()
        s = plan.stats()
        assert (s["m2l_tc_m_tiles"], s["m2l_tc_stages"], bool(s["m2l_tc_fused"])) == (mt, st, fused)
        results[(mt, st, fused)] = H
    for fused in (False, True):
        group = [H for (mt, st, f), H in results.items() if f == fused]
        for H in group[1:]:
            np.testing.assert_array_equal(H, group[0])
    unfused = next(H for (mt, st, f), H in results.items() if not f)
    fused_h = next(H for (mt, st, f), H in results.items() if f)
    assert oracle.rel_l2(fused_h, unfused) < 1e-6
    ref = oracle.fmm(x, x, m[K - 1].astype(np.float64), order, 3, identities=np.arange(n), flags=2)["H"]
    assert oracle.rel_l2(unfused[K - 1], ref) < FP32_REL_L2
    with pytest.raises(ValueError, match="not a pipeline shape"):
        plan.set_m2l_shape(3, 99, False)
    plan.set_m2l_shape(0)  # back to autotuning
    plan.evaluate(m, output="field")
    plan.close()


def clustered_6000(seed):
    """6,000 points in two Gaussian clusters (sigma 0.04) inside the unit
    cube: at depth 2 four leaves hold > 128 points, the densest ~2,500."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.3, 0.7, (2, 3))
    x = np.clip(c[rng.integers(0, 2, 6000)] + rng.normal(scale=0.04, size=(6000, 3)), 0.001, 0.999)
    return rng, x


@pytest.mark.parametrize("K", [1, 3, 8])
def test_dense_leaves_split_over_work_units(K):
    """A leaf with more than 128 targets is split into near-field work units
    of at most 128 targets (one CTA each, the heaviest first); every state
    still meets the FP32 bar against the FP64 oracle FMM, for the K = 1
    kernel, the plain K < 4 layout and the paired K >= 4 layout.  A target
    here sums up to ~7,500 near sources with strong cancellation in FP32, so
    the bar is the larger of 3e-5 and twice the reference's own FP32 error on
    the same points and states (its CpuStatic FP32 against its FP64,
    tests/golden/pins.npz)."""
    import hashlib

    g = load_group("pins.npz", "clustered_6000")
    rng, x = clustered_6000(5)
    assert hashlib.sha256(x.tobytes()).hexdigest() == str(g["sources_sha"])
    n = len(x)
    leaf = np.floor(x * 4).astype(int) @ np.array([16, 4, 1])
    assert np.bincount(leaf).max() > 4 * 128
    ms = rng.normal(size=(K, n, 3)).astype(np.float32)
    f = make_fmm(x, x, 5, 2, root=[0.5, 0.5, 0.5, 0.5], max_states=K)
    ids = np.arange(n)
    r = f.evaluate_states(ms, output="both", target_source_indices=ids.tolist())
    for k in sorted({0, K - 1}):
        key = f"K{K}_s{k}_"
        assert hashlib.sha256(ms[k].tobytes()).hexdigest() == str(g[key + "moments_sha"])
        bar_h = max(FP32_REL_L2, 2.0 * float(g[key + "ref32_rel_l2_H"]))
        bar_phi = max(FP32_REL_L2, 2.0 * float(g[key + "ref32_rel_l2_phi"]))
        assert oracle.rel_l2(r["H"][k], g[key + "H64"]) < bar_h
        assert oracle.rel_l2(r["phi"][k], g[key + "phi64"]) < bar_phi
        ref = oracle.fmm(x, x, ms[k].astype(np.float64), 5, 2, identities=ids, root_centre=[0.5, 0.5, 0.5],
                         root_half_width=0.5)
        assert oracle.rel_l2(r["H"][k], ref["H"]) < bar_h
        assert oracle.rel_l2(r["phi"][k], ref["phi"]) < bar_phi


def test_k1_near_field_does_not_depend_on_the_unit_split():
    """A K = 1 target's near-field sum runs over its leaf's neighbourhood in
    one fixed order whatever unit of its leaf it falls in: a standalone call
    (units capped by cost, 16-128 targets) and the same plan inside a batch
    graph (uncapped units of 128) give bit-identical fields.  This checks the
    work-unit cover exactly, independent of any tolerance."""
    torch = pytest.importorskip("torch")
    rng, x = clustered_6000(5)
    n = len(x)
    o = cdfmm.UniformTreeOptions()
    o.max_level = 2
    o.root_centre = cdfmm.Vec3(0.5, 0.5, 0.5)
    o.root_half_width = 0.5
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 5, max_states=1)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = torch.from_numpy(rng.normal(size=(1, n, 3)).astype(np.float32)).cuda()
    alone = torch.empty((1, n, 3), device="cuda")
    plan.evaluate(m, output="field", field=alone)
    batched = torch.empty((1, n, 3), device="cuda")
    batch = cdfmm_b200.Batch([(plan, m, batched, None)], output="field")
    batch.launch()
    np.testing.assert_array_equal(batched.cpu().numpy(), alone.cpu().numpy())
    batch.close()
    plan.close()


@pytest.mark.parametrize("K", [8, 64])
def test_near_far_schedules_give_the_same_field(K):
    """Both near/far schedules of a K-state evaluation (the full-size near
    field beside the far field; the upward pass first, then the co-resident
    near-field form beside the tensor-core M2L) compute the same sums:
    results agree to FP32 rounding (the co-resident form sums each target's
    state blocks of 32 in another order, and the M2L may take another
    pipeline shape) and meet the FP32 bar against the FP64 oracle FMM.  The
    concurrent trace reports each stream's interval in order; AUTO resolves
    to SEPARATE.  The schedules
    are those of the FP32 near field; with the tensor-core near field every
    schedule runs SEPARATE."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(400 + K)
    n = 6000
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 5, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    plan.set_near_mode(cdfmm_b200.NEAR_FP32)
    out = {}
    for sched in (cdfmm_b200.SCHEDULE_SEPARATE, cdfmm_b200.SCHEDULE_CORUN, cdfmm_b200.SCHEDULE_AUTO):
        plan.set_schedule(sched)
        H = torch.empty((K, n, 3), device="cuda")
        phi = torch.empty((K, n), device="cuda")
        plan.set_timing(2)
        plan.evaluate(m, output="both", field=H, potential=phi, synchronize=True)
        plan.set_timing(0)
        st = plan.stats()
        expect = cdfmm_b200.SCHEDULE_SEPARATE if sched == cdfmm_b200.SCHEDULE_AUTO else sched
        assert st["schedule_last"] == expect
        assert 0.0 <= st["trace_p2p_begin"] <= st["trace_p2p_end"] <= st["trace_end"]
        assert st["trace_far_begin"] <= st["trace_m2l_begin"] <= st["trace_far_end"] <= st["trace_end"]
        if expect == cdfmm_b200.SCHEDULE_CORUN:
            assert st["trace_far_begin"] <= st["trace_p2p_begin"]  # upward pass first
        out[sched] = (H.cpu().numpy(), phi.cpu().numpy())
    base_h, base_phi = out[cdfmm_b200.SCHEDULE_SEPARATE]
    for sched, (h, p) in out.items():
        assert oracle.rel_l2(h, base_h) < 1e-6
        assert oracle.rel_l2(p, base_phi) < 1e-6
    # AUTO runs SEPARATE (checked above); its M2L shape is tuned again after
    # the CORUN call's smaller budget and may take the other hi/lo fusion, so
    # the two agree to rounding (the loop above), not bit for bit
    ref = oracle.fmm(x, x, m[K - 1].cpu().numpy().astype(np.float64), 5, 3, identities=np.arange(n))
    h, p = out[cdfmm_b200.SCHEDULE_AUTO]
    assert oracle.rel_l2(h[K - 1], ref["H"]) < FP32_REL_L2
    assert oracle.rel_l2(p[K - 1], ref["phi"]) < FP32_REL_L2
    plan.set_near_mode(cdfmm_b200.NEAR_AUTO)
    plan.set_schedule(cdfmm_b200.SCHEDULE_CORUN)
    plan.evaluate(m, output="both", field=H, potential=phi, synchronize=True)
    assert plan.stats()["near_tc_last"] == 1
    assert plan.stats()["schedule_last"] == cdfmm_b200.SCHEDULE_SEPARATE
    assert oracle.rel_l2(H.cpu().numpy(), base_h) < 2e-6
    with pytest.raises(ValueError, match="unknown schedule"):
        plan.set_schedule(7)
    plan.close()


def test_results_do_not_depend_on_other_live_plans():
    """Plans created while other plans stay alive land on other memory; a
    kernel that reads past one of its own arrays would then see whatever lies
    there.  Regression of the M2L operand pack, which read its level-scale
    table past the deepest level for the zero padding (stale non-finite
    words there made every local NaN): each new plan must give the same
    finite field as the first."""
    rng = np.random.default_rng(9)
    n, K = 2000, 8
    x = rng.uniform(0, 1, (n, 3))
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    self_map = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]
    big = np.random.default_rng(10).random((50000, 3))
    mb = np.random.default_rng(11).normal(size=(1, 50000, 3))
    side = np.random.default_rng(12).random((3000, 3))
    alive, first, first_big = [], None, None
    for it in range(6):
        plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
        plan.set_self_indices(self_map)
        plan.set_m2l_shape(*plan.m2l_shapes()[0])
        H = plan.evaluate(m, output="field")["H"]
        plan.close()
        assert np.isfinite(H).all(), f"iteration {it}"
        if first is None:
            first = H
        np.testing.assert_array_equal(H, first)
        p6 = cdfmm_b200.DevicePlan.from_points(big, 6, 3)
        p6.set_m2l_shape(*p6.m2l_shapes()[0])
        Hb = p6.evaluate(mb, output="field")["H"]
        p6.close()
        assert np.isfinite(Hb).all(), f"iteration {it}"
        if first_big is None:
            first_big = Hb
        np.testing.assert_array_equal(Hb, first_big)
        # a plan of another order kept alive for the rest of the test
        alive.append(cdfmm_b200.DevicePlan.from_points(side, 5, 3))
    for p in alive:
        p.close()
