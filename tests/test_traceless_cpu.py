"""The traceless reduction the tensor-core M2L applies, checked on the CPU
against the library's own FP64 M2L matrices (cdfmm_b200_m2l_stencil).

The operator T[alpha][beta] = D^(alpha+beta) G with G = 1/(4 pi |R|) harmonic,
so every derivative tensor is traceless: D^(g+2x) + D^(g+2y) + D^(g+2z) = 0.
Folding a moment with alpha_z >= 2 onto (alpha - 2z + 2x) and
(alpha - 2z + 2y) with the sign flipped, and recovering the locals with
beta_z >= 2 from L_beta = -L_(beta-2z+2x) - L_(beta-2z+2y), the sub-block of
T on the (p+1)^2 - 1 folded moments (alpha_z <= 1, the monopole, identically
zero for dipoles, left out) and the (p+1)^2 locals with beta_z <= 1
reproduces the full product exactly in exact arithmetic.  This is the
mathematics; the GPU parity tests check the device tables and kernels."""
import numpy as np
import pytest

import cdfmm_b200


def basis(p):
    out = []
    for d in range(p + 1):
        for a in range(d + 1):
            for b in range(d - a + 1):
                out.append((a, b, d - a - b))
    return out


def rank(a, b, c):
    d = a + b + c
    return d * (d + 1) * (d + 2) // 6 + a * (d + 1) - a * (a - 1) // 2 + b


def fold(M, B, p):
    M = M.copy()
    for z in range(p, 1, -1):
        for i, (a, b, c) in enumerate(B):
            if c == z and M[i] != 0.0:
                M[rank(a + 2, b, c - 2)] -= M[i]
                M[rank(a, b + 2, c - 2)] -= M[i]
                M[i] = 0.0
    return M


def expand(L, B, p):
    L = L.copy()
    for z in range(2, p + 1):
        for i, (a, b, c) in enumerate(B):
            if c == z:
                L[i] = -(L[rank(a + 2, b, c - 2)] + L[rank(a, b + 2, c - 2)])
    return L


@pytest.mark.parametrize("p", [2, 4, 6, 8])
def test_traceless_subblock_reproduces_the_full_m2l(p):
    T, _ = cdfmm_b200.m2l_stencil(p)
    B = basis(p)
    n = len(B)
    assert all(rank(*e) == i for i, e in enumerate(B))
    ins = [i for i, e in enumerate(B) if e[2] <= 1 and i > 0]
    outs = [i for i, e in enumerate(B) if e[2] <= 1]
    assert len(ins) == (p + 1) ** 2 - 1 and len(outs) == (p + 1) ** 2
    rng = np.random.default_rng(p)
    for t in [(2, 0, 0), (-3, 1, 2), (3, 3, -3), (0, -2, 1), (1, 2, 3)]:
        slot = (t[0] + 3) * 49 + (t[1] + 3) * 7 + (t[2] + 3)
        M = rng.normal(size=n)
        M[0] = 0.0  # dipole distributions have no monopole
        full = T[slot].T @ M  # L[beta] = sum_alpha T[alpha][beta] M[alpha]
        Mf = fold(M, B, p)
        assert np.all(Mf[[i for i, e in enumerate(B) if e[2] > 1]] == 0.0)
        L = np.zeros(n)
        L[outs] = T[slot][np.ix_(ins, outs)].T @ Mf[ins]
        red = expand(L, B, p)
        assert np.abs(red - full).max() <= 1e-12 * np.abs(full).max()


def test_derivative_tensors_are_traceless():
    """The premise: D^(g+2x) + D^(g+2y) + D^(g+2z) = 0 for every entry of the
    stencil with |g| + 2 <= 2p (checked through T's first row, alpha = 0)."""
    p = 6
    T, _ = cdfmm_b200.m2l_stencil(p)
    B = basis(p)
    for slot in [(5 * 49 + 3 * 7 + 3), (0 * 49 + 6 * 7 + 2), (4 * 49 + 0 * 7 + 6)]:
        row = T[slot][0]  # D^beta G for |beta| <= p
        scale = np.abs(row).max()
        for (a, b, c) in B:
            if a + b + c + 2 <= p:
                s = row[rank(a + 2, b, c)] + row[rank(a, b + 2, c)] + row[rank(a, b, c + 2)]
                assert abs(s) <= 1e-12 * scale


@pytest.mark.parametrize("p", [0, 1, 3, 6, 8, 10])
def test_library_tables_match_the_restatement(p):
    """The tables the device kernels use (cdfmm_b200_m2l_traceless) against
    this file's restatement: the same input and output sets, each folded
    moment the same signed sum (its own rank first, coefficient 1), and the
    derived locals in an order where both sources come first; applied to
    the library's FP64 operators they reproduce the full product."""
    t = cdfmm_b200.m2l_traceless(p)
    B = basis(p)
    n = len(B)
    ins = [i for i, e in enumerate(B) if e[2] <= 1 and i > 0]
    outs = [i for i, e in enumerate(B) if e[2] <= 1]
    assert list(t["in"]) == ins and list(t["out"]) == outs
    # fold: column j of the CSR equals the restated fold of every moment
    F = np.zeros((len(ins), n))
    for j in range(len(ins)):
        lo, hi = t["fold_offsets"][j], t["fold_offsets"][j + 1]
        assert t["fold_ranks"][lo] == ins[j] and t["fold_coefficients"][lo] == 1
        for r, c in zip(t["fold_ranks"][lo:hi], t["fold_coefficients"][lo:hi]):
            F[j, r] += c
    for a in range(1, n):
        e = np.zeros(n)
        e[a] = 1.0
        np.testing.assert_array_equal(F[:, a], fold(e, B, p)[ins])
    # derived locals: sources computed before use, z lowered by two
    known = set(outs)
    for d, s1, s2 in t["derived"]:
        assert s1 in known and s2 in known and d not in known
        a, b, c = B[d]
        assert (s1, s2) == (rank(a + 2, b, c - 2), rank(a, b + 2, c - 2))
        known.add(int(d))
    assert known == set(range(n))
    if p >= 2:
        T, _ = cdfmm_b200.m2l_stencil(p)
        rng = np.random.default_rng(10 + p)
        slot = 1 * 49 + 5 * 7 + 3
        M = rng.normal(size=n)
        M[0] = 0.0
        L = np.zeros(n)
        L[outs] = T[slot][np.ix_(ins, outs)].T @ (F @ M)
        for d, s1, s2 in t["derived"]:
            L[d] = -(L[s1] + L[s2])
        full = T[slot].T @ M
        assert np.abs(L - full).max() <= 1e-12 * np.abs(full).max()
