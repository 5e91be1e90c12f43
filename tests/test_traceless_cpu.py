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
