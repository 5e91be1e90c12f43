"""C ABI and host-layer checks that need no GPU.

- the library loads and exports every function include/cdfmm_b200.h declares;
- the plan's M2L matrices (host FP64 generation) match the reference's
  (tests/golden/m2l_matrices.npz; upstream tests/test_static_m2l.cpp:330-355);
- argument validation maps to the reference's exception types;
- without a device, plan creation fails with ERR_NO_DEVICE (no CPU fallback).
"""

import ctypes
import os
import re

import numpy as np
import pytest

import cdfmm
import cdfmm_b200
from conftest import GOLDEN, ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "cdfmm_b200.h")).read()
    return sorted(set(re.findall(r"\b(cdfmm_b200_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = cdfmm_b200.library()
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(cdfmm_b200.EXPORTED)


def test_plan_m2l_matrices_match_reference():
    data = np.load(os.path.join(GOLDEN, "m2l_matrices.npz"))
    for key in data.files:
        p_str, off = key.split("__")
        p = int(p_str[1:])
        if off == "phys":
            R = np.array([0.55, 0.3, -0.4]) - np.array([0.1, -0.2, 0.05])
        else:
            R = np.array([float(v) for v in off.split("_")])
        ours = cdfmm_b200.m2l_matrix(p, R)
        ref = data[key]
        np.testing.assert_allclose(ours, ref, rtol=1e-12, atol=4e-13 * np.abs(ref).max(), err_msg=key)


def test_m2l_matrix_argument_errors():
    with pytest.raises(ValueError):
        cdfmm_b200.m2l_matrix(3, [0.0, 0.0, 0.0])
    with pytest.raises(ValueError):
        cdfmm_b200.m2l_matrix(11, [2.0, 0.0, 0.0])


def test_plan_creation_without_device_fails_loudly():
    if cdfmm_b200.device_count() > 0:
        pytest.skip("a device is present")
    x = np.random.default_rng(0).uniform(0, 1, (100, 3))
    o = cdfmm.UniformTreeOptions()
    o.max_level = 2
    t = cdfmm.UniformTree(x, x, o)
    with pytest.raises(cdfmm_b200.CdfmmError) as err:
        cdfmm_b200.DevicePlan.from_tree(t, 4)
    assert err.value.code == cdfmm_b200.ERR_NO_DEVICE
    opts = cdfmm.UniformFmmOptions()
    opts.tree.max_level = 2
    with pytest.raises(RuntimeError, match="no CUDA device"):
        cdfmm.UniformFmm(x, x, opts)


def test_option_validation_matches_reference_exceptions():
    x = np.random.default_rng(1).uniform(0, 1, (10, 3))
    o = cdfmm.UniformFmmOptions()
    o.expansion_order = -1
    with pytest.raises(ValueError, match="expansion_order must be >= 0"):
        cdfmm.UniformFmm(x, o)
    o = cdfmm.UniformFmmOptions()
    o.backend = cdfmm.ExecutionBackend.CPU_STATIC
    with pytest.raises(RuntimeError, match="unavailable in this build"):
        cdfmm.UniformFmm(x, x, o)
    o = cdfmm.UniformFmmOptions()
    o.precision = cdfmm.StaticPrecision.FLOAT64
    with pytest.raises(ValueError, match="FP32"):
        cdfmm.UniformFmm(x, x, o)
    o = cdfmm.UniformFmmOptions()
    o.fixed_target_source_indices = [0, 1]
    with pytest.raises(ValueError, match="one entry per target"):
        cdfmm.UniformFmm(x, x, o)
    o.fixed_target_source_indices = list(range(9)) + [10]
    with pytest.raises(ValueError, match="invalid source index"):
        cdfmm.UniformFmm(x, x, o)


def test_enum_and_alias_compatibility():
    assert cdfmm.ExecutionBackend.CUDA_M2L == cdfmm.ExecutionBackend.CUDA_M2L_P2P
    assert cdfmm.ExecutionBackend.CUDA_M2L_STATIC_P2P == cdfmm.ExecutionBackend.CUDA_M2L_P2P
    assert cdfmm.cuda_m2l_available() == cdfmm.cuda_m2l_p2p_available()
    o = cdfmm.UniformFmmOptions()
    assert o.precision == cdfmm.StaticPrecision.FLOAT32
    assert o.static_matrix_backend == cdfmm.StaticMatrixBackend.PORTABLE
    assert len(cdfmm.multi_indices(6)) == 84
    assert cdfmm.multi_indices(1) == [[0, 0, 0], [0, 0, 1], [0, 1, 0], [1, 0, 0]]
