"""Tensor-core near field (cdfmm_b200_set_near_mode): TF32 hi/lo pair-tensor
products against the FP32 SIMT near field and the FP64 direct sum.

The near field is the reference's list-1 P2P (upstream src/operators.cpp:
178-199 pair formula, src/uniform_tree.cpp:455-480 neighbourhood); the
tensor-core form must give the same sums at FP32-level accuracy: against the
FP64 direct sum on a depth-1 tree (every pair is a near pair) it must be as
accurate as the FP32 form, and on deeper trees it must agree with the FP32
form to rounding level."""
import numpy as np
import pytest

import cdfmm_b200
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _evaluate(plan, m, mode, output="both"):
    plan.set_near_mode(mode)
    K, n = m.shape[0], plan.n_targets
    H = torch.full((K, n, 3), float("nan"), dtype=torch.float32, device="cuda")
    phi = torch.full((K, n), float("nan"), dtype=torch.float32, device="cuda")
    plan.evaluate(m, output=output, field=H, potential=phi, synchronize=True)
    return H.cpu().numpy(), phi.cpu().numpy(), plan.stats()["near_tc_last"]


def _points(kind, n, rng):
    if kind == "uniform":
        return rng.uniform(0, 1, (n, 3))
    c = rng.uniform(0.2, 0.8, (4, 3))
    return c[rng.integers(0, 4, n)] + rng.normal(0, 0.03, (n, 3))


@pytest.mark.parametrize("kind", ["uniform", "clusters"])
def test_near_field_alone_is_as_accurate_as_fp32(kind):
    """Depth 1: the FMM is the near field alone.  Both forms against the FP64
    direct sum (FP32 moments), every state checked on two of them."""
    rng = np.random.default_rng(11)
    n, K = 3000, 8
    x = _points(kind, n, rng)
    plan = cdfmm_b200.DevicePlan.from_points(x, 4, 1, max_states=K)
    mm = rng.normal(size=(K, n, 3)).astype(np.float32)
    m = torch.from_numpy(mm).cuda()
    H32, p32, used32 = _evaluate(plan, m, cdfmm_b200.NEAR_FP32)
    Htc, ptc, usedtc = _evaluate(plan, m, cdfmm_b200.NEAR_TF32X3)
    assert (used32, usedtc) == (0, 1)
    ids = np.arange(n, dtype=np.int32)
    for k in (0, K - 1):
        phi64, H64 = cdfmm_b200.direct_fp64(x, mm[k].astype(np.float64), x, ids)
        e32, etc = oracle.rel_l2(H32[k], H64), oracle.rel_l2(Htc[k], H64)
        assert etc < 2e-6 and etc < 2.0 * e32, (etc, e32)
        assert oracle.rel_l2(ptc[k], phi64) < 2e-6
    plan.close()


@pytest.mark.parametrize("K", [8, 24, 64])
def test_tensor_core_and_fp32_near_fields_agree(K):
    """Depth 3 (far field present): the two near-field forms give the same
    field and potential to rounding level for K rounded up to 16 (padding
    states), and the result meets the FP32 bar against the FP64 oracle FMM
    (same tree and order: the truncation error of p = 4 cancels)."""
    rng = np.random.default_rng(100 + K)
    n = 20000
    x = rng.uniform(0, 1, (n, 3))
    plan = cdfmm_b200.DevicePlan.from_points(x, 4, 3, max_states=K)
    m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    H32, p32, _ = _evaluate(plan, m, cdfmm_b200.NEAR_FP32)
    Htc, ptc, used = _evaluate(plan, m, cdfmm_b200.NEAR_AUTO)
    assert used == 1
    assert oracle.rel_l2(Htc, H32) < 2e-6
    assert oracle.rel_l2(ptc, p32) < 2e-6
    k = K - 1
    ref = oracle.fmm(x, x, m[k].cpu().numpy().astype(np.float64), 4, 3, identities=np.arange(n))
    assert oracle.rel_l2(Htc[k], ref["H"]) < 3e-5
    assert oracle.rel_l2(ptc[k], ref["phi"]) < 3e-5
    plan.close()


def test_dense_neighbourhoods_and_separate_targets():
    """Clustered points at depth 2: some neighbourhoods hold more than the
    1,536 sources whose positions are staged in shared memory (the kernel
    then reads them from global memory), and targets distinct from the
    sources (no self pairs)."""
    rng = np.random.default_rng(5)
    ns, nt, K = 40000, 3000, 16
    src = 0.5 + rng.normal(0, 0.06, (ns, 3))
    tgt = 0.5 + rng.normal(0, 0.08, (nt, 3))
    plan = cdfmm_b200.DevicePlan.from_points(src, 4, 2, targets=tgt, root_centre=(0.5, 0.5, 0.5),
                                             root_half_width=0.6, max_states=K)
    tree = plan.tree()
    counts = np.diff(tree["leaf_source_offsets"])
    assert counts.max() > 1536
    m = torch.from_numpy(rng.normal(size=(K, ns, 3)).astype(np.float32)).cuda()
    H32, p32, _ = _evaluate(plan, m, cdfmm_b200.NEAR_FP32)
    Htc, ptc, used = _evaluate(plan, m, cdfmm_b200.NEAR_TF32X3)
    assert used == 1 and np.isfinite(Htc).all()
    assert oracle.rel_l2(Htc, H32) < 2e-6
    assert oracle.rel_l2(ptc, p32) < 2e-6
    plan.close()


def test_field_only_output_and_state_range():
    """Field-only output leaves the potential untouched by the near field;
    K outside 8..64 keeps the FP32 near field."""
    rng = np.random.default_rng(3)
    n = 5000
    x = rng.uniform(0, 1, (n, 3))
    plan = cdfmm_b200.DevicePlan.from_points(x, 4, 2, max_states=72)
    m8 = torch.from_numpy(rng.normal(size=(8, n, 3)).astype(np.float32)).cuda()
    Hf, _, used = _evaluate(plan, m8, cdfmm_b200.NEAR_AUTO, output="field")
    Hb, _, _ = _evaluate(plan, m8, cdfmm_b200.NEAR_AUTO, output="both")
    assert used == 1
    np.testing.assert_array_equal(Hf, Hb)
    for K in (4, 72):
        m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
        _, _, used = _evaluate(plan, m, cdfmm_b200.NEAR_AUTO)
        assert used == 0
    plan.close()


def test_near_field_expired_waits_poison_and_recover():
    """With the SIMT M2L (no tensor-core far field) and the injected wait
    limit 0, the tensor-core near field's progress waits expire: the call
    reports a timeout and its near-field targets read NaN; with the default
    limit restored the next evaluation equals the one before."""
    rng = np.random.default_rng(21)
    n, K = 4000, 16
    x = rng.uniform(0, 1, (n, 3))
    plan = cdfmm_b200.DevicePlan.from_points(x, 4, 3, max_states=K, m2l_mode=cdfmm_b200.M2L_FP32)
    plan.set_near_mode(cdfmm_b200.NEAR_TF32X3)
    m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    H = torch.empty((K, n, 3), dtype=torch.float32, device="cuda")
    plan.evaluate(m, output="field", field=H, synchronize=True)
    clean = H.cpu().numpy().copy()
    assert np.isfinite(clean).all()
    plan.set_wait_limit(0)
    with pytest.raises(cdfmm_b200.CdfmmError) as err:
        plan.evaluate(m, output="field", field=H, synchronize=True)
    assert err.value.code == cdfmm_b200.ERR_TIMEOUT
    assert np.isnan(H.cpu().numpy()).any()
    plan.poll_status()
    plan.set_wait_limit(-1)
    plan.evaluate(m, output="field", field=H, synchronize=True)
    np.testing.assert_array_equal(H.cpu().numpy(), clean)
    plan.close()


def test_set_near_mode_rejects_unknown_modes():
    rng = np.random.default_rng(1)
    plan = cdfmm_b200.DevicePlan.from_points(rng.uniform(0, 1, (100, 3)), 2, 1, max_states=8)
    with pytest.raises(ValueError, match="unknown near-field mode"):
        plan.set_near_mode(7)
    plan.close()


@pytest.mark.parametrize("kind", ["uniform", "clusters"])
def test_position_gradient_on_tensor_cores(kind):
    """The backward's near-field position gradient on the tensor cores
    (X = sum_k w_k m_k^T per pair as one matrix product over the states):
    on a depth-1 tree (every pair near) against the FP64 direct gradient
    summed over the states, within 3x the FP32 kernel's error and below
    2e-6, and against the FP32 kernel to rounding level.  The moment
    gradient (transposed evaluation) is unchanged by the near-field form up
    to rounding."""
    rng = np.random.default_rng(3)
    n, K = 3000, 8
    x = _points(kind, n, rng)
    plan = cdfmm_b200.DevicePlan.from_points(x, 4, 1, max_states=K)
    mm = rng.normal(size=(K, n, 3)).astype(np.float32)
    ww = rng.normal(size=(K, n, 3)).astype(np.float32)
    m, w = torch.from_numpy(mm).cuda(), torch.from_numpy(ww).cuda()
    out = {}
    for mode in (cdfmm_b200.NEAR_FP32, cdfmm_b200.NEAR_TF32X3):
        plan.set_near_mode(mode)
        gx = torch.full((n, 3), float("nan"), dtype=torch.float32, device="cuda")
        gm = torch.full((K, n, 3), float("nan"), dtype=torch.float32, device="cuda")
        plan.backward(w, moments=m, grad_moments=gm, grad_target_positions=gx, want_moments=True,
                      want_positions=True, synchronize=True)
        out[mode] = (gx.cpu().numpy(), gm.cpu().numpy())
    ids = np.arange(n, dtype=np.int32)
    ref = sum(cdfmm_b200.direct_grad_fp64(x, mm[k].astype(np.float64), x, ww[k].astype(np.float64), ids)
              for k in range(K))
    g32, gtc = out[cdfmm_b200.NEAR_FP32][0], out[cdfmm_b200.NEAR_TF32X3][0]
    e32, etc = oracle.rel_l2(g32, ref), oracle.rel_l2(gtc, ref)
    assert np.isfinite(gtc).all()
    assert etc < 2e-6 and etc < 3.0 * e32, (etc, e32)
    assert oracle.rel_l2(gtc, g32) < 2e-6
    assert oracle.rel_l2(out[cdfmm_b200.NEAR_TF32X3][1], out[cdfmm_b200.NEAR_FP32][1]) < 2e-6
    plan.close()


def test_tensor_core_forms_across_state_counts_and_point_sets():
    """One plan (max 64 states) called with K = 17 (padded to 32 MMA
    columns), 64 and 8 in turn, targets distinct from the sources, depth 3
    (neighbourhood positions staged in shared memory): field, potential and
    position gradient of both near-field forms agree to rounding level on
    every call."""
    rng = np.random.default_rng(29)
    ns, nt = 15000, 4000
    src = rng.uniform(0, 1, (ns, 3))
    tgt = rng.uniform(0, 1, (nt, 3))
    plan = cdfmm_b200.DevicePlan.from_points(src, 4, 3, targets=tgt, root_centre=(0.5, 0.5, 0.5),
                                             root_half_width=0.5, max_states=64)
    for K in (17, 64, 8):
        m = torch.from_numpy(rng.normal(size=(K, ns, 3)).astype(np.float32)).cuda()
        w = torch.from_numpy(rng.normal(size=(K, nt, 3)).astype(np.float32)).cuda()
        res = {}
        for mode in (cdfmm_b200.NEAR_FP32, cdfmm_b200.NEAR_TF32X3):
            H, phi, used = _evaluate(plan, m, mode)
            assert used == (1 if mode == cdfmm_b200.NEAR_TF32X3 else 0)
            gx = torch.full((nt, 3), float("nan"), dtype=torch.float32, device="cuda")
            plan.backward(w, moments=m, grad_target_positions=gx, want_moments=False, want_positions=True,
                          synchronize=True)
            res[mode] = (H, phi, gx.cpu().numpy())
        a, b = res[cdfmm_b200.NEAR_FP32], res[cdfmm_b200.NEAR_TF32X3]
        assert np.isfinite(b[0]).all() and np.isfinite(b[2]).all()
        assert oracle.rel_l2(b[0], a[0]) < 2e-6, K
        assert oracle.rel_l2(b[1], a[1]) < 2e-6, K
        assert oracle.rel_l2(b[2], a[2]) < 2e-6, K
    plan.close()


@pytest.mark.parametrize("order,K", [(4, 8), (6, 16), (7, 64)])
def test_tensor_core_p2m_matches_fp32_p2m(order, K):
    """With the near field on the tensor cores its packed moment blocks also
    feed the leaf multipoles (tensor-core P2M, orders <= 7): every node's
    multipoles (leaves and, through M2M, every level above) agree with the
    FP32 P2M's to TF32 hi/lo rounding, relative to the node's largest
    coefficient, for the first and last state; the two are not bit-identical
    (the tensor-core form ran)."""
    rng = np.random.default_rng(200 + K)
    n = 30000
    x = rng.uniform(0, 1, (n, 3))
    plan = cdfmm_b200.DevicePlan.from_points(x, order, 3, max_states=K)
    m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    _, _, used32 = _evaluate(plan, m, cdfmm_b200.NEAR_FP32)
    M32 = [plan.read_expansions("multipole", k).astype(np.float64) for k in (0, K - 1)]
    _, _, usedtc = _evaluate(plan, m, cdfmm_b200.NEAR_AUTO)
    Mtc = [plan.read_expansions("multipole", k).astype(np.float64) for k in (0, K - 1)]
    plan.close()
    assert (used32, usedtc) == (0, 1)
    for a, b in zip(M32, Mtc):
        assert np.all(np.isfinite(b))
        scale = np.abs(a).max(axis=1)
        err = np.abs(a - b).max(axis=1)
        assert np.all(err <= 1e-5 * scale + 1e-30), float((err / np.maximum(scale, 1e-30)).max())
        assert not np.array_equal(a, b)
