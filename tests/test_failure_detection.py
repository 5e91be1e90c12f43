"""Failure detection without a GPU fault.

Every wait of the tensor-core M2L pipeline on an mbarrier is bounded: on
expiry the kernel records an error code in a device flag, stops issuing,
drains and returns, and the host turns the flag into
CDFMM_B200_ERR_TIMEOUT.  The self-test entry point runs a kernel whose wait
cannot complete (nothing arrives on the barrier) with a short limit; the
test checks the status, the message, and that the device context is still
usable by running a normal evaluation right after.  Host-side failures
(bad arguments, missing device) are covered by the ABI tests.
"""

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
import oracle

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_with_timeout_status_and_context_survives():
    lib = cdfmm_b200.library()
    rc = lib.cdfmm_b200_selftest_bounded_wait(0)
    assert rc == cdfmm_b200.ERR_TIMEOUT
    assert "expired as intended" in lib.cdfmm_b200_last_error(None).decode()
    # the context is intact: an evaluation on the tensor-core path works
    rng = np.random.default_rng(8)
    n, K = 2000, 8
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = rng.normal(size=(K, n, 3)).astype(np.float32)
    H = plan.evaluate(m, output="field")["H"]
    assert plan.stats()["m2l_mode_resolved"] == cdfmm_b200.M2L_BF16X3
    ref = oracle.fmm(x, x, m[3].astype(np.float64), 4, 3, identities=np.arange(n), flags=2)["H"]
    assert oracle.rel_l2(H[3], ref) < 3e-5
    plan.close()


def test_selftest_rejects_bad_device():
    lib = cdfmm_b200.library()
    assert lib.cdfmm_b200_selftest_bounded_wait(10_000) == cdfmm_b200.ERR_INVALID_ARGUMENT


def test_async_expired_wait_poisons_results_and_is_reported_once():
    """An asynchronous tensor-core evaluate whose progress waits are made to
    expire at once (injected limit 0, no fault): its results are NaN, not the
    previous call's values; a later synchronous call on the plan reports only
    its own status; poll_status reports the asynchronous failure once; with
    the default limit restored the next evaluation is clean and equal to the
    one before the failure."""
    import torch

    rng = np.random.default_rng(9)
    n, K = 2000, 8
    x = rng.uniform(0, 1, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 3
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, 4, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    m = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    H = torch.empty((K, n, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    plan.evaluate(m, output="field", field=H, stream=stream, synchronize=True)  # tunes the M2L shape
    assert plan.stats()["m2l_mode_resolved"] == cdfmm_b200.M2L_BF16X3
    clean = H.cpu().numpy().copy()
    assert np.isfinite(clean).all()
    plan.poll_status()  # nothing pending

    plan.set_wait_limit(0)
    plan.evaluate(m, output="field", field=H, stream=stream, synchronize=False)
    torch.cuda.synchronize()
    poisoned = H.cpu().numpy()
    assert np.isnan(poisoned).all(), "every far field passes through an aborted M2L tile"
    # a synchronous call that itself expires reports its own timeout
    with pytest.raises(cdfmm_b200.CdfmmError) as own:
        plan.evaluate(m, output="field", field=H, stream=stream, synchronize=True)
    assert own.value.code == cdfmm_b200.ERR_TIMEOUT and "this call" in str(own.value)
    assert "1 earlier call" in str(own.value)
    plan.poll_status()  # both failures were reported by the synchronous call

    # an asynchronous failure followed by a clean synchronous call: the clean
    # call succeeds; poll_status then reports the earlier failure, once
    plan.evaluate(m, output="field", field=H, stream=stream, synchronize=False)
    plan.set_wait_limit(-1)
    plan.evaluate(m, output="field", field=H, stream=stream, synchronize=True)
    np.testing.assert_array_equal(H.cpu().numpy(), clean)
    with pytest.raises(cdfmm_b200.CdfmmError) as late:
        plan.poll_status()
    assert late.value.code == cdfmm_b200.ERR_TIMEOUT and "1 call(s)" in str(late.value)
    plan.poll_status()
    ref = oracle.fmm(x, x, m[2].cpu().numpy().astype(np.float64), 4, 3, identities=np.arange(n), flags=2)["H"]
    assert oracle.rel_l2(clean[2], ref) < 3e-5
    plan.close()
