"""Pins the CPU oracle (oracle/oracle.c) against the reference's own outputs.

Golden vectors come from the upstream reference (tests/golden/make_golden.py).
Tolerances follow the reference's own tests where they exist:
M2L matrices vs the reference builder (tests/test_static_m2l.cpp:330-355 uses
eps 4e-13), FP64 FMM vs FP64 reference (rel 1e-10 here: different derivative
method and summation order), direct sum (1e-13).
"""

import numpy as np
import pytest

import oracle
from conftest import group_names, load_group


@pytest.mark.parametrize("name", group_names("trees.npz"))
def test_oracle_tree_matches_reference(name):
    g = load_group("trees.npz", name)
    root = g["root_in"]
    has_root = bool(g["has_root"])
    t = oracle.tree(g["sources"], g["targets"], int(g["depth"]),
                    root[:3] if has_root else None, root[3] if has_root else None)
    np.testing.assert_array_equal(t["source_permutation"], g["source_permutation"])
    np.testing.assert_array_equal(t["target_permutation"], g["target_permutation"])
    np.testing.assert_array_equal(t["ranges"], g["ranges"])
    np.testing.assert_array_equal(t["root_centre"], g["root_centre"])
    assert t["root_half_width"] == g["root_half_width"]


@pytest.mark.parametrize("depth", [2, 3])
def test_oracle_lists_match_reference(depth):
    data = np.load(f"{oracle._HERE}/../tests/golden/lists.npz")
    l1o, l1, l2o, l2 = oracle.lists(depth)
    np.testing.assert_array_equal(l1o, data[f"d{depth}__l1_off"])
    np.testing.assert_array_equal(l1, data[f"d{depth}__l1"])
    np.testing.assert_array_equal(l2o, data[f"d{depth}__l2_off"])
    np.testing.assert_array_equal(l2, data[f"d{depth}__l2"])


def test_oracle_m2l_matrices_match_reference():
    data = np.load(f"{oracle._HERE}/../tests/golden/m2l_matrices.npz")
    for key in data.files:
        p_str, off = key.split("__")
        p = int(p_str[1:])
        if off == "phys":
            R = np.array([0.55, 0.3, -0.4]) - np.array([0.1, -0.2, 0.05])
        else:
            R = np.array([float(v) for v in off.split("_")])
        ours = oracle.m2l_matrix(p, R)
        ref = data[key]
        scale = np.abs(ref).max()
        np.testing.assert_allclose(ours, ref, rtol=1e-12, atol=4e-13 * scale, err_msg=key)


def test_oracle_pair_known_answers():
    # upstream tests/test_p2p.cpp:13-33: axial H.x = 2c, transverse H.x = -c
    c = 1.0 / (4.0 * np.pi)
    _, H = oracle.direct([[0, 0, 0]], [[1, 0, 0]], [[1, 0, 0]])
    np.testing.assert_allclose(H[0], [2 * c, 0, 0], atol=1e-15)
    _, H = oracle.direct([[0, 0, 0]], [[1, 0, 0]], [[0, 1, 0]])
    np.testing.assert_allclose(H[0], [-c, 0, 0], atol=1e-15)


@pytest.mark.parametrize("name", group_names("fmm.npz"))
def test_oracle_direct_matches_reference(name):
    g = load_group("fmm.npz", name)
    ids = g["identities"] if g["identities"].size else None
    phi, H = oracle.direct(g["sources"], g["moments"], g["targets"], ids)
    np.testing.assert_allclose(H, g["H_direct"], rtol=1e-12, atol=1e-12 * np.abs(g["H_direct"]).max())
    np.testing.assert_allclose(phi, g["phi_direct"], rtol=1e-12, atol=1e-12 * np.abs(g["phi_direct"]).max())


@pytest.mark.parametrize("name", group_names("fmm.npz"))
def test_oracle_fmm_matches_reference_fp64(name):
    g = load_group("fmm.npz", name)
    ids = g["identities"] if g["identities"].size else None
    root = g["root_in"]
    has_root = bool(g["has_root"])
    r = oracle.fmm(g["sources"], g["targets"], g["moments"], int(g["order"]), int(g["depth"]), ids, 3,
                   root[:3] if has_root else None, root[3] if has_root else None)
    assert oracle.rel_l2(r["H"], g["H64"]) < 1e-10
    assert oracle.rel_l2(r["phi"], g["phi64"]) < 1e-10
    # depth 0 is exactly the direct sum (upstream tests/test_uniform_fmm.cpp:429-451)
    if int(g["depth"]) == 0:
        np.testing.assert_allclose(r["H"], g["H_direct"], rtol=1e-14, atol=1e-14 * np.abs(g["H_direct"]).max())


def test_oracle_expansions_match_reference_fp32():
    g = load_group("fmm.npz", "expansions_p4_d3")
    r = oracle.fmm(g["sources"], g["targets"], g["moments"], 4, 3, g["identities"], 3, expansions=True)
    t = oracle.tree(g["sources"], g["targets"], 3)
    s = 2.0 * t["root_half_width"]
    deg = oracle.basis(4).sum(axis=1)
    M_norm = r["M"] * s ** (-(deg + 2.0))
    L_norm = r["L"] * s ** (deg - 1.0)
    for ours, ref in ((M_norm, g["M32"].astype(np.float64)), (L_norm, g["L32"].astype(np.float64))):
        scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
        assert np.max(np.abs(ours - ref) / scale) < 2e-5
