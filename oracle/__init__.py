"""CPU oracle for the static-geometry uniform dipole FMM (test infrastructure).

This package restates upstream dip-fmm's UniformFmm::evaluate path in FP64 C
(oracle/oracle.c, built into oracle/liboracle.so by oracle/Makefile) and wraps
it with numpy.  It is the CHECKER: only tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs use it.  The product
(dip-fmm_b200/) never imports it.

Parity of this restatement is pinned against golden vectors produced by the
upstream reference itself (tests/golden/make_golden.py, run against the
reference sources compiled by oracle/ref.mk), see tests/test_oracle_golden.py.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def library() -> ctypes.CDLL:
    """Loads (building on first use if needed) oracle/liboracle.so."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i, i64 = ctypes.c_double, ctypes.c_int, ctypes.c_int64
    lib.oracle_basis_size.argtypes = [i]
    lib.oracle_basis_size.restype = i
    lib.oracle_basis.argtypes = [i, P(i)]
    lib.oracle_laplace_derivatives.argtypes = [i, P(d), P(d)]
    lib.oracle_m2l_matrix.argtypes = [i, P(d), P(d)]
    lib.oracle_tree.argtypes = [i, P(d), i, P(d), i, i, P(d), i, d, P(d), P(i), P(i), P(i64)]
    lib.oracle_tree.restype = i
    lib.oracle_lists.argtypes = [i, P(i), P(i), P(i), P(i)]
    lib.oracle_direct.argtypes = [i, P(d), P(d), i, P(d), P(i), i, P(d), P(d)]
    lib.oracle_direct_grad.argtypes = [i, P(d), P(d), i, P(d), P(i), P(d), P(d)]
    lib.oracle_cuboid_tensor.argtypes = [P(d), P(d), P(d)]
    lib.oracle_cuboid_monomial.argtypes = [i, i, i, P(d), P(d)]
    lib.oracle_cuboid_monomial.restype = d
    lib.oracle_direct_cuboid.argtypes = [i, P(d), P(d), P(d), i, i, P(d), P(d), P(d)]
    lib.oracle_fmm.argtypes = [i, P(d), i, P(d), i, i, i, P(d), d, P(d), P(i), i, P(d), P(d), P(d), P(d)]
    lib.oracle_fmm.restype = i
    _LIB = lib
    return lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def level_offset(level: int) -> int:
    return ((1 << (3 * level)) - 1) // 7


def basis(p: int) -> np.ndarray:
    lib = library()
    n = lib.oracle_basis_size(p)
    out = np.zeros((n, 3), dtype=np.int32)
    lib.oracle_basis(p, _ip(out))
    return out


def laplace_derivatives(order: int, R) -> np.ndarray:
    lib = library()
    out = np.zeros(lib.oracle_basis_size(order))
    lib.oracle_laplace_derivatives(order, _dp(_f64(R)), _dp(out))
    return out


def m2l_matrix(p: int, R) -> np.ndarray:
    """(n, n) matrix with [beta, alpha] = D^{alpha+beta} G(R)."""
    lib = library()
    n = lib.oracle_basis_size(p)
    out = np.zeros(n * n)
    lib.oracle_m2l_matrix(p, _dp(_f64(R)), _dp(out))
    return out.reshape(n, n).T.copy()  # stored [beta + n*alpha]


def tree(sources, targets, depth, root_centre=None, root_half_width=None):
    lib = library()
    s, t = _f64(sources).reshape(-1, 3), _f64(targets).reshape(-1, 3)
    nodes = level_offset(depth + 1)
    root = np.zeros(4)
    sp = np.zeros(len(s), dtype=np.int32)
    tp = np.zeros(len(t), dtype=np.int32)
    ranges = np.zeros((nodes, 4), dtype=np.int64)
    c = _f64(root_centre if root_centre is not None else [0, 0, 0])
    rc = lib.oracle_tree(len(s), _dp(s), len(t), _dp(t), depth, int(root_centre is not None), _dp(c),
                         int(root_half_width is not None), float(root_half_width or 0.0), _dp(root),
                         _ip(sp), _ip(tp), ranges.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    if rc != 0:
        raise ValueError("Point lies outside the requested root box")
    return {"root_centre": root[:3], "root_half_width": root[3], "source_permutation": sp,
            "target_permutation": tp, "ranges": ranges}


def lists(depth: int):
    lib = library()
    nodes = level_offset(depth + 1)
    l1o = np.zeros(nodes + 1, dtype=np.int32)
    l2o = np.zeros(nodes + 1, dtype=np.int32)
    l1 = np.zeros(nodes * 27, dtype=np.int32)
    l2 = np.zeros(nodes * 189, dtype=np.int32)
    lib.oracle_lists(depth, _ip(l1o), _ip(l1), _ip(l2o), _ip(l2))
    return l1o, l1[: l1o[-1]], l2o, l2[: l2o[-1]]


def direct(sources, moments, targets, self_indices=None, flags=3):
    """FP64 O(N*M) direct sum; returns (phi, H)."""
    lib = library()
    s, m, t = _f64(sources).reshape(-1, 3), _f64(moments).reshape(-1, 3), _f64(targets).reshape(-1, 3)
    phi = np.zeros(len(t))
    H = np.zeros((len(t), 3))
    ids = _i32(self_indices)
    lib.oracle_direct(len(s), _dp(s), _dp(m), len(t), _dp(t), _ip(ids), flags, _dp(phi), _dp(H))
    return phi, H


def direct_grad(sources, moments, targets, weights, self_indices=None):
    """FP64 direct gradient of L = sum_i w_i . H_i w.r.t. the target positions."""
    lib = library()
    s, m, t = _f64(sources).reshape(-1, 3), _f64(moments).reshape(-1, 3), _f64(targets).reshape(-1, 3)
    w = _f64(weights).reshape(-1, 3)
    g = np.zeros((len(t), 3))
    lib.oracle_direct_grad(len(s), _dp(s), _dp(m), len(t), _dp(t), _ip(_i32(self_indices)), _dp(w), _dp(g))
    return g


def fmm(sources, targets, moments, order, depth, identities=None, flags=3, root_centre=None,
        root_half_width=None, expansions=False):
    """FP64 uniform FMM in physical units; returns dict(phi, H[, M, L])."""
    lib = library()
    s, t, m = _f64(sources).reshape(-1, 3), _f64(targets).reshape(-1, 3), _f64(moments).reshape(-1, 3)
    n = lib.oracle_basis_size(order)
    nodes = level_offset(depth + 1)
    phi = np.zeros(len(t))
    H = np.zeros((len(t), 3))
    M = np.zeros((nodes, n)) if expansions else None
    L = np.zeros((nodes, n)) if expansions else None
    has_root = root_centre is not None
    c = _f64(root_centre if has_root else [0, 0, 0])
    rc = lib.oracle_fmm(len(s), _dp(s), len(t), _dp(t), order, depth, int(has_root), _dp(c),
                        float(root_half_width or 0.0), _dp(m), _ip(_i32(identities)), flags, _dp(phi),
                        _dp(H), _dp(M), _dp(L))
    if rc != 0:
        raise ValueError("Point lies outside the requested root box")
    out = {"phi": phi, "H": H}
    if expansions:
        out["M"], out["L"] = M, L
    return out


def cuboid_tensor(r, h) -> np.ndarray:
    """(3, 3) [field][moment] field per unit total moment of a uniformly
    magnetised cuboid of side lengths h at r from its centre."""
    out = np.zeros(9)
    library().oracle_cuboid_tensor(_dp(_f64(r)), _dp(_f64(h)), _dp(out))
    return out.reshape(3, 3)


def cuboid_monomial(alpha, d, h) -> float:
    """(d + u)^alpha / alpha! averaged over u in the cuboid of side lengths h."""
    return library().oracle_cuboid_monomial(int(alpha[0]), int(alpha[1]), int(alpha[2]), _dp(_f64(d)), _dp(_f64(h)))


def direct_cuboid(sources, moments, sizes, targets):
    """FP64 direct sum over cuboid sources: (phi, H) at the targets."""
    s, m, t = _f64(sources), _f64(moments), _f64(targets)
    h = _f64(sizes).reshape(-1, 3)
    phi = np.zeros(len(t))
    H = np.zeros((len(t), 3))
    library().oracle_direct_cuboid(len(s), _dp(s), _dp(m), _dp(h), len(h), len(t), _dp(t), _dp(phi), _dp(H))
    return phi, H


def rel_l2(a, b) -> float:
    """sqrt(sum |a-b|^2 / sum |b|^2) (upstream tests/test_precision.cpp:21-31)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))
