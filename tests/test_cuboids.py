"""Uniformly magnetised cuboid sources (SourceGeometry.UNIFORM_CUBOID).

Pinned to the upstream reference (tests/golden/cuboids.npz, made by
tests/golden/make_cuboids.py from the reference's own module):
  - the oracle's closed-form cuboid -> point tensor against the reference's
    FP64 DenseDirectPlan (inside, on faces, edges and corners, near, far);
  - the oracle's cuboid direct sum against the reference's FP64 dense direct
    sum; the cuboid-averaged monomial against quadrature;
  - (GPU) complete evaluations of cdfmm.UniformFmm with cuboid sources
    against the reference's CpuStatic FP32 results of the same inputs
    (common and per-source sizes, with and without the cuboid P2M, touching
    cubes), the cuboid multipoles per node, and the near field alone
    (depth 0) against the oracle's FP64 direct sum.
"""

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
import oracle
from conftest import GOLDEN

FP32_REL_L2 = 3e-5
CASES = ["common_p6_d3", "common_point_p2m_p6_d3", "per_source_p5_d3", "touching_cubes_p6_d3"]


def golden():
    return np.load(f"{GOLDEN}/cuboids.npz")


def case(name):
    g = golden()
    return {k[len(name) + 2:]: g[k] for k in g.files if k.startswith(name + "__")}


def cuboid_fmm(c, max_states=1, depth=None):
    o = cdfmm.UniformFmmOptions()
    o.expansion_order = int(c["order"])
    o.tree.max_level = int(c["depth"]) if depth is None else depth
    o.max_states = max_states
    o.source_geometry = cdfmm.SourceGeometry.UNIFORM_CUBOID
    o.source_sizes = [cdfmm.CuboidSize(*map(float, h)) for h in c["sizes"]]
    o.use_cuboid_p2m = bool(c["cuboid_p2m"])
    return cdfmm.UniformFmm(c["sources"], c["sources"], o)


# ---------------------------------------------------------------- CPU -------

@pytest.mark.parametrize("shape", ["cube", "slab", "rod"])
def test_oracle_cuboid_tensor_matches_reference(shape):
    g = golden()
    h = g[f"tensor__{shape}__h"]
    T_ref = g[f"tensor__{shape}__T"]
    # each of the 8 corner terms is O(1 / V): far away their sum cancels to
    # O(h^3 / r^3), so both FP64 evaluations carry ~1e-16 / V of rounding
    atol = 1e-13 / h.prod()
    for r, Tr in zip(g[f"tensor__{shape}__targets"], T_ref):
        T = oracle.cuboid_tensor(r, h)
        np.testing.assert_allclose(T, Tr, rtol=1e-12, atol=atol)
        np.testing.assert_allclose(T, T.T, rtol=0, atol=0)


def test_oracle_cube_self_field_and_far_limit():
    h = np.array([0.3, 0.3, 0.3])
    np.testing.assert_allclose(oracle.cuboid_tensor([0, 0, 0], h) * h.prod(), -np.eye(3) / 3.0, atol=1e-15)
    r = np.array([4.0, -3.0, 7.5])
    rn = np.linalg.norm(r)
    point = (3 * np.outer(r, r) / rn**5 - np.eye(3) / rn**3) / (4 * np.pi)
    # a cube's first correction is of degree 4 in h / r (the degree-2 term cancels)
    np.testing.assert_allclose(oracle.cuboid_tensor(r, h), point, rtol=0, atol=1e-6 * np.abs(point).max())


def test_oracle_cuboid_monomial_against_quadrature():
    x, w = np.polynomial.legendre.leggauss(8)
    d = np.array([0.31, -0.12, 0.07])
    h = np.array([0.2, 0.5, 0.15])
    from math import factorial

    for alpha in [(0, 0, 0), (2, 0, 1), (3, 2, 0), (1, 1, 4), (0, 5, 2), (6, 0, 0)]:
        q = 1.0
        for a in range(3):
            u = 0.5 * h[a] * x
            q *= 0.5 * np.sum(w * (d[a] + u) ** alpha[a]) / factorial(alpha[a])
        assert abs(oracle.cuboid_monomial(alpha, d, h) - q) <= 1e-14 * max(abs(q), 1e-300)


@pytest.mark.parametrize("name", CASES)
def test_oracle_cuboid_direct_matches_reference(name):
    c = case(name)
    phi, H = oracle.direct_cuboid(c["sources"], c["moments"], c["sizes"], c["sources"])
    assert oracle.rel_l2(H, c["H_direct"]) < 1e-12
    assert oracle.rel_l2(phi, c["phi_direct"]) < 1e-12


def test_cuboid_option_checks():
    x = np.random.default_rng(1).random((20, 3))
    o = cdfmm.UniformFmmOptions()
    o.tree.max_level = 1
    o.source_sizes = [cdfmm.CuboidSize(0.1, 0.1, 0.1)]
    with pytest.raises(ValueError, match="point-dipole sources do not accept cuboid sizes"):
        cdfmm.UniformFmm(x, x, o)
    o.source_geometry = cdfmm.SourceGeometry.UNIFORM_CUBOID
    o.source_sizes = [cdfmm.CuboidSize(0.1, 0.1, 0.1)] * 3
    with pytest.raises(ValueError, match="cuboid sizes must contain one or one per source"):
        cdfmm.UniformFmm(x, x, o)


# ---------------------------------------------------------------- GPU -------

@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_cuboid_evaluate_matches_reference_cpustatic(name):
    c = case(name)
    f = cuboid_fmm(c)
    r = f.evaluate(c["moments"], output="both")
    # the same truncated expansion as the reference's FP32 plan
    assert oracle.rel_l2(r["H"], c["H32"]) < FP32_REL_L2
    assert oracle.rel_l2(r["phi"], c["phi32"]) < FP32_REL_L2
    # and as close to the exact (FP64 dense direct) field as the reference
    ref_err = oracle.rel_l2(c["H64"], c["H_direct"])
    assert oracle.rel_l2(r["H"], c["H_direct"]) < ref_err + FP32_REL_L2
    # identities do not apply to cuboid sources (their self fields are physical)
    r2 = f.evaluate(c["moments"], output="both", target_source_indices=list(range(len(c["sources"]))))
    np.testing.assert_array_equal(r["H"], r2["H"])


@pytest.mark.gpu
def test_cuboid_multipoles_match_reference():
    c = case("common_p6_d3")
    f = cuboid_fmm(c)
    f.evaluate(c["moments"])
    nn = len(f.tree.nodes)
    M = np.stack([f.multipole(i) for i in range(nn)]).astype(np.float64)
    ref = c["M32"].astype(np.float64)
    scale = np.abs(ref).max(axis=1)
    assert np.all(np.abs(M - ref).max(axis=1) <= 2e-5 * scale + 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["per_source_p5_d3", "touching_cubes_p6_d3"])
def test_cuboid_near_field_alone_matches_oracle(name):
    """Depth 0: every pair is a list-1 pair, so the result is the near field
    alone: the FP32-stored FP64 tensors against the oracle's FP64 sum."""
    c = case(name)
    x, m, h = c["sources"][:1500], c["moments"][:1500], c["sizes"]
    h = h if len(h) == 1 else h[:1500]
    o = cdfmm.UniformFmmOptions()
    o.expansion_order = 2
    o.tree.max_level = 0
    o.source_geometry = cdfmm.SourceGeometry.UNIFORM_CUBOID
    o.source_sizes = [cdfmm.CuboidSize(*map(float, v)) for v in h]
    f = cdfmm.UniformFmm(x, x, o)
    r = f.evaluate(m, output="both")
    phi, H = oracle.direct_cuboid(x, m, h, x)
    assert oracle.rel_l2(r["H"], H) < 2e-6
    assert oracle.rel_l2(r["phi"], phi) < 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("K", [3, 8, 20])
def test_cuboid_states_batched_like_single_calls(K):
    c = case("per_source_p5_d3")
    rng = np.random.default_rng(K)
    m = rng.normal(size=(K, len(c["sources"]), 3)) * 1e-3
    f = cuboid_fmm(c, max_states=K)
    r = f.evaluate_states(m.astype(np.float32), output="both")
    g = cuboid_fmm(c)
    for k in (0, K - 1):
        s = g.evaluate(m[k], output="both")
        assert oracle.rel_l2(r["H"][k], s["H"]) < 2e-6
        assert oracle.rel_l2(r["phi"][k], s["phi"]) < 2e-6


@pytest.mark.gpu
def test_cuboid_plan_api():
    c = case("common_p6_d3")
    x, m = c["sources"], c["moments"][None]
    t = cdfmm.UniformTree(x, x, _tree_options(3))
    plan = cdfmm_b200.DevicePlan.from_tree(t, 6, max_states=1)
    plan.set_self_indices(np.array(t.source_inverse_permutation)[np.array(t.target_permutation)])
    point = plan.evaluate(m, output="both")
    plan.set_source_cuboids(c["sizes"][0], cuboid_p2m=True)
    cub = plan.evaluate(m, output="both")
    assert oracle.rel_l2(cub["H"][0], c["H32"]) < FP32_REL_L2
    with pytest.raises(ValueError, match="dimensions must be positive"):
        plan.set_source_cuboids([0.1, 0.0, 0.1])
    with pytest.raises(cdfmm_b200.CdfmmError, match="point-dipole sources only"):
        plan.backward(np.ones((1, len(x), 3), np.float32), m.astype(np.float32))
    plan.set_source_cuboids(None)
    again = plan.evaluate(m, output="both")
    np.testing.assert_array_equal(point["H"], again["H"])
    np.testing.assert_array_equal(point["phi"], again["phi"])
    plan.close()


def _tree_options(depth):
    o = cdfmm.UniformTreeOptions()
    o.max_level = depth
    return o
