"""Multi-geometry batches: several independent geometries of uneven size
(clustered points, depth per problem for ~32 points per leaf) evaluated by one
CUDA graph launch through cdfmm_b200_batch_*.

Each geometry's result must equal that plan's own cdfmm_b200_evaluate
bit for bit (the graph replays the same kernels) -- or, for one-state plans
whose M2L the batch stacks with others of the same depth and order into one
tensor-core M2L, agree with it to FP32 rounding -- and match the FP64 oracle
FMM of that geometry within the FP32 tolerance; a relaunch after the inputs
change in place must follow them.
"""

import math

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
import oracle

pytestmark = pytest.mark.gpu


def clustered_points(rng, n, clusters=8, sigma=0.05):
    """n points from `clusters` isotropic Gaussians (centres U[0.1, 0.9]^3),
    points outside the unit cube rejected and redrawn."""
    centres = rng.uniform(0.1, 0.9, (clusters, 3))
    out = np.empty((0, 3))
    while len(out) < n:
        c = centres[rng.integers(0, clusters, size=2 * n)]
        p = c + rng.normal(scale=sigma, size=c.shape)
        p = p[np.all((p >= 0.0) & (p < 1.0), axis=1)]
        out = np.concatenate([out, p])
    return out[:n]


def depth_for(n):
    return max(1, int(round(math.log(n / 32.0, 8))))


def _problem(rng, n, order, K):
    x = clustered_points(rng, n)
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth_for(n)
    tree = cdfmm.UniformTree(x, x, o)
    plan = cdfmm_b200.DevicePlan.from_tree(tree, order, max_states=K)
    plan.set_self_indices(np.array(tree.source_inverse_permutation)[np.array(tree.target_permutation)])
    d = rng.normal(size=(K, n, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    return x, plan, d.astype(np.float32)


@pytest.mark.parametrize("K", [1, 8])
def test_batch_matches_individual_evaluations_and_oracle(K):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024 + K)
    sizes = [700, 2048, 5000, 9000, 16384, 3000]
    order = 4
    probs, items = [], []
    for n in sizes:
        x, plan, m = _problem(rng, n, order, K)
        dm = torch.from_numpy(m).cuda()
        dH = torch.full((K, n, 3), float("nan"), device="cuda")
        probs.append((x, plan, m, dm, dH))
        items.append((plan, dm, dH, None))
    batch = cdfmm_b200.Batch(items, output="field")
    groups = batch.groups()
    if K == 1:  # depths 2 and 3 hold several one-state problems each: stacked
        assert sum(g >= 0 for g in groups) >= 4 and len({g for g in groups if g >= 0}) == 2
    else:
        assert all(g < 0 for g in groups)
    for rnd in range(2):
        if rnd == 1:  # new moments in place: the graph reads the same buffers
            for x, plan, m, dm, dH in probs:
                m *= -0.5
                dm.copy_(torch.from_numpy(m))
                dH.fill_(float("nan"))
        batch.launch()
        torch.cuda.synchronize()
        for (x, plan, m, dm, dH), g in zip(probs, groups):
            got = dH.cpu().numpy()
            ref = plan.evaluate(m, output="field")["H"]
            if g < 0:
                np.testing.assert_array_equal(got, ref)
            else:
                assert oracle.rel_l2(got, ref) < 2e-6
            o64 = oracle.fmm(x, x, m[0].astype(np.float64), order, depth_for(len(x)), identities=np.arange(len(x)),
                             flags=2)["H"]
            assert oracle.rel_l2(got[0], o64) < 3e-5
    batch.close()
    for x, plan, m, dm, dH in probs:
        plan.close()


def test_batch_argument_errors():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x, plan, m = _problem(rng, 1000, 3, 1)
    dm = torch.from_numpy(m).cuda()
    dH = torch.zeros((1, 1000, 3), device="cuda")
    with pytest.raises(ValueError, match="once per batch"):
        cdfmm_b200.Batch([(plan, dm, dH, None), (plan, dm, dH, None)])
    with pytest.raises(ValueError, match="device-resident"):
        a = cdfmm_b200.EvalArgs()
        a.moments = cdfmm_b200._ptr(m).value
        a.n_states = 1
        a.output = cdfmm_b200.OUTPUT_FIELD
        a.field = cdfmm_b200._ptr(dH).value
        a.memory = cdfmm_b200.MOMENTS_ON_HOST
        import ctypes
        plans = (ctypes.c_void_p * 1)(plan._h.value)
        args = (cdfmm_b200.EvalArgs * 1)(a)
        h = ctypes.c_void_p()
        cdfmm_b200._check(cdfmm_b200.library().cdfmm_b200_batch_create(plans, args, 1, ctypes.byref(h)))
    plan.close()
