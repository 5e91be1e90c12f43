"""Reverse mode: dL/dmoments and dL/dtarget-positions of L = sum_k sum_i w_ik . H_ik.

The reference has no reverse mode; these tests pin ours three ways:
  * dL/dm is the exact transpose of the evaluated FMM: <w, A m> = <A^t w, m>
    to FP32 rounding (the linear map's own finite difference), and it matches
    the FP64 direct-sum transpose (the field of the weights at the sources,
    sources and targets exchanged) to the FMM's FP32 tolerance;
  * dL/dx_target matches the FP64 direct-sum gradient (oracle.direct_grad)
    and a central finite difference (h = 1e-4) of the evaluated FMM along a
    random direction (targets that would change leaf are held still);
  * the torch.autograd.Function gives the same gradients as the C ABI.
The CPU test checks oracle.direct_grad itself against finite differences of
oracle.direct.
"""

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
import oracle


def _tree(src, tgt, depth, root=None):
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth
    if root is not None:
        o.root_centre = cdfmm.Vec3(*root[:3])
        o.root_half_width = float(root[3])
    return cdfmm.UniformTree(src, tgt, o)


def _plan(src, tgt, order, depth, K, self_map=True, m2l=cdfmm_b200.M2L_AUTO, root=None):
    tree = _tree(src, tgt, depth, root)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, order, max_states=K, m2l_mode=m2l)
    if self_map:
        sorted_self = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]
        plan.set_self_indices(sorted_self)
    return plan


def _dipoles(rng, K, n):
    d = rng.normal(size=(K, n, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    return d * rng.uniform(0.5, 1.5, size=(K, n, 1))


def test_oracle_direct_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    src = rng.uniform(0, 1, (300, 3))
    tgt = rng.uniform(0, 1, (40, 3))
    m = rng.normal(size=(300, 3))
    w = rng.normal(size=(40, 3))
    g = oracle.direct_grad(src, m, tgt, w)
    h = 1e-5
    fd = np.zeros_like(tgt)
    for c in range(3):
        tp, tm = tgt.copy(), tgt.copy()
        tp[:, c] += h
        tm[:, c] -= h
        Hp = oracle.direct(src, m, tp, flags=2)[1]
        Hm = oracle.direct(src, m, tm, flags=2)[1]
        fd[:, c] = np.sum(w * (Hp - Hm), axis=1) / (2 * h)
    assert oracle.rel_l2(g, fd) < 1e-5  # O(h^2) truncation of the difference quotient


@pytest.mark.parametrize("same_points", [True, False])
@pytest.mark.parametrize("order,depth", [(3, 4), (4, 3), (6, 2)])
def test_swapped_fmm_is_the_exact_transpose_in_fp64(same_points, order, depth):
    # The identity the transposed plan rests on, in the FP64 oracle:
    # <w, FMM(sources -> targets) m> = <FMM(targets -> sources) w, m>.
    rng = np.random.default_rng(3 + order)
    n = 1500
    src = rng.uniform(0, 1, (n, 3))
    tgt = src if same_points else rng.uniform(0, 1, (1100, 3))
    m = rng.normal(size=(n, 3))
    w = rng.normal(size=(len(tgt), 3))
    ids = np.arange(n) if same_points else None
    H = oracle.fmm(src, tgt, m, order, depth, identities=ids, flags=2)["H"]
    G = oracle.fmm(tgt, src, w, order, depth, identities=ids, flags=2)["H"]
    lhs, rhs = np.sum(w * H), np.sum(G * m)
    assert abs(lhs - rhs) < 1e-13 * np.sum(np.abs(w * H))


@pytest.mark.gpu
@pytest.mark.parametrize("K,m2l", [(1, cdfmm_b200.M2L_FP32), (8, cdfmm_b200.M2L_AUTO), (8, cdfmm_b200.M2L_FP32)])
@pytest.mark.parametrize("same_points", [True, False])
def test_grad_moments_is_the_exact_transpose(K, m2l, same_points):
    rng = np.random.default_rng(100 + K + 7 * int(same_points))
    n = 4096
    src = rng.uniform(0, 1, (n, 3))
    tgt = src if same_points else rng.uniform(0, 1, (3000, 3))
    plan = _plan(src, tgt, 4, 3, K, self_map=same_points, m2l=m2l)
    m = _dipoles(rng, K, n).astype(np.float32)
    w = rng.normal(size=(K, len(tgt), 3)).astype(np.float32)
    H = plan.evaluate(m, output="field")["H"]
    gm = plan.backward(w, want_moments=True)["moments"]
    assert gm.shape == m.shape and np.all(np.isfinite(gm))
    lhs = float(np.sum(w.astype(np.float64) * H))
    rhs = float(np.sum(gm.astype(np.float64) * m))
    scale = float(np.sum(np.abs(w.astype(np.float64) * H)))
    assert abs(lhs - rhs) < 2e-6 * scale, (lhs, rhs, scale)
    # The same FMM with sources and targets exchanged, in FP64 (the oracle):
    # equal to FP32 rounding.  Against the FP64 direct-sum transpose (the
    # weights' field at the sources): within the p = 4 truncation error.
    self_t = np.arange(n) if same_points else None
    for k in range(K):
        ref_fmm = oracle.fmm(tgt, src, w[k], 4, 3, identities=self_t, flags=2)["H"]
        assert oracle.rel_l2(gm[k], ref_fmm) < 1e-5
        ref = oracle.direct(tgt, w[k], src, self_t, flags=2)[1]
        assert oracle.rel_l2(gm[k], ref) < 5e-4
    plan.close()


@pytest.mark.gpu
@pytest.mark.parametrize("order,K", [(6, 1), (6, 4), (8, 8)])
def test_grad_positions_match_fp64_direct_gradient(order, K):
    rng = np.random.default_rng(300 + order + K)
    n = 4096
    x = rng.uniform(0, 1, (n, 3))
    plan = _plan(x, x, order, 3, K)
    m = _dipoles(rng, K, n)
    w = rng.normal(size=(K, n, 3))
    g = plan.backward(w.astype(np.float32), moments=m, want_moments=False, want_positions=True)["positions"]
    ref = np.zeros((n, 3))
    for k in range(K):
        ref += oracle.direct_grad(x, m[k], x, w[k], np.arange(n))
    err = oracle.rel_l2(g, ref)
    assert err < (2e-4 if order == 6 else 5e-5), err
    plan.close()


@pytest.mark.gpu
def test_grad_positions_match_central_finite_differences():
    rng = np.random.default_rng(404)
    n, depth, order, K = 4096, 3, 6, 2
    root = (0.5, 0.5, 0.5, 0.5)
    x = rng.uniform(0.01, 0.99, (n, 3))
    m = _dipoles(rng, K, n).astype(np.float32)
    w = rng.normal(size=(K, n, 3)).astype(np.float32)
    h = 1e-4
    # Targets that move are those farther than 1e-3 from a leaf face (they
    # keep their leaf) and 1e-2 from every other point (the central
    # difference's O(h^2 / r^2) error stays below ~1e-3; the closest pairs of
    # 4096 uniform points are ~1e-3 apart, where it would reach 100%).
    cell = (x - (np.array(root[:3]) - root[3])) / (2 * root[3]) * (1 << depth)
    frac = cell - np.floor(cell)
    width = 2 * root[3] / (1 << depth)
    safe = np.all((frac * width > 1e-3) & ((1 - frac) * width > 1e-3), axis=1)
    d2 = np.sum((x[:, None, :] - x[None, :, :]) ** 2, axis=2)
    np.fill_diagonal(d2, np.inf)
    safe &= d2.min(axis=1) > 1e-4
    v = rng.normal(size=(n, 3)) * safe[:, None]

    def loss(tgt):
        plan = _plan(x, tgt, order, depth, K, root=root)
        H = plan.evaluate(m, output="field")["H"]
        plan.close()
        return float(np.sum(w.astype(np.float64) * H))

    fd = (loss(x + h * v) - loss(x - h * v)) / (2 * h)
    plan = _plan(x, x, order, depth, K, root=root)
    g = plan.backward(w, moments=m, want_moments=False, want_positions=True)["positions"]
    plan.close()
    analytic = float(np.sum(g.astype(np.float64) * v))
    assert abs(fd - analytic) < 2e-3 * abs(analytic), (fd, analytic)


@pytest.mark.gpu
def test_autograd_function_matches_c_abi():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    n, K = 4096, 4
    x = rng.uniform(0, 1, (n, 3))
    plan = _plan(x, x, 6, 3, K)
    m_np = _dipoles(rng, K, n).astype(np.float32)
    w_np = rng.normal(size=(K, n, 3)).astype(np.float32)
    m = torch.tensor(m_np, device="cuda", requires_grad=True)
    xt = torch.tensor(x, dtype=torch.float32, device="cuda", requires_grad=True)
    w = torch.tensor(w_np, device="cuda")
    H = cdfmm_b200.dipole_field(plan, m, xt)
    (w * H).sum().backward()
    torch.cuda.synchronize()
    # the backward reused the forward's sorted moments and leaf locals
    assert plan.stats()["backward_reused_forward"] == 1
    ref = plan.backward(w_np, moments=m_np, want_moments=True, want_positions=True)
    H_ref = plan.evaluate(m_np, output="field")["H"]
    np.testing.assert_allclose(H.detach().cpu().numpy(), H_ref, rtol=0, atol=1e-6 * np.abs(H_ref).max())
    gm = m.grad.cpu().numpy()
    gx = xt.grad.cpu().numpy()
    np.testing.assert_allclose(gm, ref["moments"], rtol=0, atol=1e-6 * np.abs(ref["moments"]).max())
    np.testing.assert_allclose(gx, ref["positions"], rtol=0, atol=1e-6 * np.abs(ref["positions"]).max())
    plan.close()


@pytest.mark.gpu
def test_backward_argument_errors():
    rng = np.random.default_rng(9)
    x = rng.uniform(0, 1, (512, 3))
    plan = _plan(x, x, 4, 2, 2)
    w = np.zeros((2, 512, 3), dtype=np.float32)
    with pytest.raises(ValueError, match="grad_moments and/or"):
        plan.backward(w, want_moments=False, want_positions=False)
    with pytest.raises(ValueError, match="forward moments"):
        plan.backward(w, want_moments=False, want_positions=True)
    with pytest.raises(ValueError, match="n_states"):
        plan.backward(np.zeros((3, 512, 3), dtype=np.float32))
    # a self map naming one source twice has no transpose plan
    tree = _tree(x, x, 2)
    bad = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]
    bad[1] = bad[0]
    plan.set_self_indices(bad)
    with pytest.raises(ValueError, match="one-to-one"):
        plan.backward(w)
    plan.close()


@pytest.mark.gpu
def test_device_fp64_direct_gradient_matches_oracle():
    rng = np.random.default_rng(77)
    src = rng.uniform(0, 1, (3000, 3))
    tgt = rng.uniform(0, 1, (500, 3))
    m = rng.normal(size=(3000, 3))
    w = rng.normal(size=(500, 3))
    self_idx = rng.integers(-1, 3000, size=500).astype(np.int32)
    g = cdfmm_b200.direct_grad_fp64(src, m, tgt, w, self_idx)
    ref = oracle.direct_grad(src, m, tgt, w, self_idx)
    assert oracle.rel_l2(g, ref) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("K", [1, 8])
def test_grad_over_dense_leaves(K):
    """Two Gaussian clusters at depth 2 (leaves of up to ~2,500 points, split
    into near-field work units of at most 128 targets): dL/dm is still the
    exact transpose and dL/dx matches the FP64 direct-sum gradient."""
    rng = np.random.default_rng(606 + K)
    c = rng.uniform(0.3, 0.7, (2, 3))
    x = np.clip(c[rng.integers(0, 2, 6000)] + rng.normal(scale=0.04, size=(6000, 3)), 0.001, 0.999)
    n = len(x)
    plan = _plan(x, x, 6, 2, K, root=[0.5, 0.5, 0.5, 0.5])
    m = _dipoles(rng, K, n)
    w = rng.normal(size=(K, n, 3))
    H = plan.evaluate(m.astype(np.float32), output="field")["H"]
    g = plan.backward(w.astype(np.float32), moments=m, want_moments=True, want_positions=True)
    lhs = float(np.sum(w * H))
    rhs = float(np.sum(g["moments"].astype(np.float64) * m))
    assert abs(lhs - rhs) < 2e-6 * float(np.sum(np.abs(w * H))), (lhs, rhs)
    ref = np.zeros((n, 3))
    for k in range(K):
        ref += oracle.direct_grad(x, m[k], x, w[k], np.arange(n))
    assert oracle.rel_l2(g["positions"], ref) < 2e-4
    plan.close()
