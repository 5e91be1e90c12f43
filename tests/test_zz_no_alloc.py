"""The allocation-free entry point, cdfmm_b200_evaluate_noalloc.

Some callers cannot allocate device memory while they evaluate: a framework
whose memory pool already owns the GPU's memory, a program that reserves all
its device memory up front, or a real-time loop that cannot afford the
allocator's implicit synchronisation.  They create the plan once and then evaluate
through this entry point, whose scratch lives in a fixed 64 MiB device array
compiled into the library.

These tests call it through the C ABI and check that its results equal those
of cdfmm_b200_evaluate, on two calls in a row (the shared array keeps the
previous call's contents, so the second call must not depend on them), and
that a request needing more scratch than the array holds is refused.  This
file is collected last so a failure here never hides another test's result.
"""

import ctypes

import numpy as np
import pytest

import cdfmm
import cdfmm_b200

pytestmark = pytest.mark.gpu


def _plan(n, order, depth, max_states, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.0, (n, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, order, max_states=max_states)
    sorted_self = np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)]
    plan.set_self_indices(sorted_self)
    return plan, rng


@pytest.mark.parametrize("K", [1, 8])
def test_noalloc_matches_evaluate_on_two_calls(K):
    torch = pytest.importorskip("torch")
    n = 4096
    plan, rng = _plan(n, 4, 3, K, 1234 + K)
    moments = torch.from_numpy(rng.normal(size=(K, n, 3)).astype(np.float32)).cuda()
    ref_H = torch.zeros((K, n, 3), dtype=torch.float32, device="cuda")
    ref_phi = torch.zeros((K, n), dtype=torch.float32, device="cuda")
    plan.evaluate(moments, output="both", field=ref_H, potential=ref_phi)
    torch.cuda.synchronize()
    ref_H, ref_phi = ref_H.cpu().numpy(), ref_phi.cpu().numpy()
    for call in range(2):
        H = torch.full((K, n, 3), float("nan"), dtype=torch.float32, device="cuda")
        phi = torch.full((K, n), float("nan"), dtype=torch.float32, device="cuda")
        plan.evaluate_noalloc(moments, H, phi, output="both")
        torch.cuda.synchronize()
        H, phi = H.cpu().numpy(), phi.cpu().numpy()
        np.testing.assert_allclose(H, ref_H, rtol=1e-6, atol=1e-6 * np.abs(ref_H).max(), err_msg=f"call {call}")
        np.testing.assert_allclose(phi, ref_phi, rtol=1e-6, atol=1e-6 * np.abs(ref_phi).max(), err_msg=f"call {call}")
    plan.close()


def test_noalloc_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    n = 50000
    # p = 8, depth 5: two states need ~100 MB of expansions, beyond 64 MiB.
    plan, rng = _plan(n, 8, 5, 2, 77)
    moments = torch.zeros((2, n, 3), dtype=torch.float32, device="cuda")
    H = torch.zeros((2, n, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="bytes of scratch"):
        plan.evaluate_noalloc(moments, H)
    with pytest.raises(ValueError, match="device-resident"):
        a = cdfmm_b200.EvalArgs()
        a.memory = cdfmm_b200.MOMENTS_ON_HOST
        a.n_states = 1
        a.output = cdfmm_b200.OUTPUT_FIELD
        cdfmm_b200._check(cdfmm_b200.library().cdfmm_b200_evaluate_noalloc(plan._h, ctypes.byref(a)), plan._h)
    plan.close()
