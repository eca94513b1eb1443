"""CPU checks of the CRT form (Ozaki scheme II): the moduli, the exactness of the FP64
reconstruction the kernel and the restatement share, that the scaling shifts bound every row's
2-norm (tightly), the restatement's accuracy against the compensated Dot2 reference, and that the
library derives the same norm bounds as the oracle."""
from __future__ import annotations

import math
import random

import numpy as np
import pytest


def test_moduli_pairwise_coprime_and_byte_sized(oracle_mod):
    mods = oracle_mod.CRT_MODULI
    assert len(mods) == oracle_mod.CRT_MAX and max(mods) == 256 and min(mods) > 128
    for i in range(len(mods)):
        for j in range(i):
            assert math.gcd(mods[i], mods[j]) == 1


def _sym(x: int, m: int) -> int:
    r = x % m
    if m == 256:
        return r - 256 if r >= 128 else r
    return r - m if r > m // 2 else r


@pytest.mark.parametrize("n", [8, 10, 11, 13, 15, 16, 17, 20])
def test_reconstruction_is_exact(oracle_mod, n):
    """With residues r_l in [0, m_l) (what the product stores), the limb sums started from
    K_k = -128 sum_l P_lk (+128 in limb 0) stay below 2^53, and Q = rint(L_hi F_hi + L_lo F_lo) is
    exact for every integer below Mprod (1 - 2^-20) / 2 in magnitude (the bound the scaling
    guarantees); values at the edges and every residue at its extremes included."""
    c = oracle_mod.crt_constants(n)
    Mp, mods, nl, w = c["Mprod"], [int(m) for m in c["mods"]], c["nl"], c["w"]
    edge = Mp * (2 ** 20 - 1) // 2 ** 21
    rng = random.Random(n)
    xs = [0, 1, -1, edge, -edge, edge - 1, -edge + 1] + [rng.randrange(-edge, edge + 1) for _ in range(400)]
    xs += [rng.randrange(-2 ** 40, 2 ** 40) for _ in range(100)]
    Kc = [-128.0 * float(sum(int(c["P"][l][k]) for l in range(n))) + (128.0 if k == 0 else 0.0) for k in range(nl)]
    for x in xs:
        res = [x % m for m in mods]
        L = list(Kc)
        for l in range(n):
            for k in range(nl):
                L[k] = float(res[l]) * float(c["P"][l][k]) + L[k]  # exact: the products and sums are integers
                assert abs(L[k]) < 2.0 ** 53
        Lint = sum(int(L[k]) << (w * k) for k in range(nl))
        Q = round(L[nl - 1] * c["f_hi"] + L[nl - 2] * c["f_lo"])
        assert Lint - Q * Mp == x
    # limb sums at their extremes: every residue 0 (most negative) or m - 1 (largest)
    for r in (0, None):
        L = list(Kc)
        for l in range(n):
            for k in range(nl):
                L[k] += float(mods[l] - 1 if r is None else r) * float(c["P"][l][k])
                assert abs(L[k]) < 2.0 ** 53


def test_norm_bounds_respect_the_modulus_product(oracle_mod):
    for n in range(oracle_mod.CRT_MIN, oracle_mod.CRT_MAX + 1):
        c = oracle_mod.crt_constants(n)
        Mp, ta, tb = c["Mprod"], c["ta"], c["tb"]
        assert ta <= 62 and tb <= 62 and abs(ta - tb) <= 1
        assert 2 ** (ta + tb) * 2 ** 21 <= Mp * (2 ** 20 - 1)
        if tb < 62:  # the largest such exponent sum
            assert 2 ** (ta + tb + 1) * 2 ** 21 > Mp * (2 ** 20 - 1)


def _rows(rng, K):
    """Rows of every kind the bound has to handle."""
    u = rng.uniform(-1, 1, K)
    yield u
    yield u * np.exp2(rng.integers(-60, 61, K))                # wide exponent spread
    yield u * 2.0 ** -1070                                       # subnormal and tiny normal entries
    yield np.where(rng.random(K) < 0.9, 0.0, u)                  # mostly zero
    yield u * 2.0 ** 1000                                        # near the top of the range
    v = u.copy()
    v[: K // 2] *= 2.0 ** -700                                   # chunks at very different scales
    yield v
    w = np.zeros(K)
    w[K - 1] = -0.5                                              # a single power of two, last chunk
    yield w


@pytest.mark.parametrize("chunk", [512, 128])
@pytest.mark.parametrize("K", [1, 5, 127, 129, 511, 512, 513, 1500, 4096])
def test_shift_bounds_the_row_norm_tightly(oracle_mod, K, chunk):
    """trunc(a 2^s) has 2-norm at most 2^t for every t the form uses, and above 2^(t-1.5) (the bound
    loses less than one bit to rounding the square root up to a power of two, plus the 15-bit
    mantissa bounds and ceilings), whatever the chunk length; all-zero rows take s = 0 and non-finite
    rows the sentinel."""
    rng = np.random.default_rng(K)
    L = oracle_mod.lib()
    for t in (31, 47, 54, 58, 62):
        for row in _rows(rng, K):
            row = np.ascontiguousarray(row)
            s = L.oracle_crt_shift(oracle_mod._p(row), 1, K, t, chunk)
            V = [math.trunc(math.ldexp(float(x), s)) for x in row]
            norm2 = sum(v * v for v in V)
            assert norm2 <= 4 ** t, (K, t, s)
            if np.any(np.abs(row) >= 2.0 ** -1022):
                assert norm2 > 2.0 ** (2 * t - 3), (K, t, s, math.log2(norm2) / 2)
    z = np.zeros(K)
    assert L.oracle_crt_shift(oracle_mod._p(z), 1, K, 50, chunk) == 0
    z[K // 2] = np.nan
    assert L.oracle_crt_shift(oracle_mod._p(z), 1, K, 50, chunk) == 0x7FFFFFFF


def test_column_shifts_are_row_shifts_of_the_transpose(oracle_mod):
    """Columns of B are chunked by 128 entries, rows of A by 512; otherwise the same bound."""
    rng = np.random.default_rng(5)
    B = rng.uniform(-1, 1, (1300, 9)) * np.exp2(rng.integers(-40, 41, (1300, 9)))
    sa, sb = oracle_mod.crt_shifts(np.ascontiguousarray(B.T), B, 14)
    c = oracle_mod.crt_constants(14)
    L = oracle_mod.lib()
    cols = [np.ascontiguousarray(B[:, j]) for j in range(9)]
    assert np.array_equal(sb, [L.oracle_crt_shift(oracle_mod._p(x), 1, 1300, c["tb"], 128) for x in cols])
    assert np.array_equal(sa, [L.oracle_crt_shift(oracle_mod._p(x), 1, 1300, c["ta"], 512) for x in cols])


def test_library_constants_match_the_oracle(oracle_mod):
    import libthom_b200 as lt

    for n in range(oracle_mod.CRT_MIN, oracle_mod.CRT_MAX + 1):
        c = oracle_mod.crt_constants(n)
        ta, tb, mods = lt.ozaki_crt_info(n)
        assert (ta, tb) == (c["ta"], c["tb"]), n
        assert mods == list(oracle_mod.CRT_MODULI[:n])
    L = lt.lib()
    assert L.lt_ozaki_crt_info(7, None, None, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_crt_info(21, None, None, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(None, None, None, 4, 4, 4, 1.0, 0.0, 15, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(0x1000, 0x1000, 0x1000, 4, 4, 4, 1.0, 0.0, 7, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(0x1000, 0x1000, 0x1000, 4, 4, 9_000_000, 1.0, 0.0, 15, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_crt_workspace_size(8192, 8192, 8192, 15) > 15 * 3 * 8192 * 8192


@pytest.mark.parametrize("phi,smax,n_fp64", [(0, 0, 14), (8, 0, 14), (32, 0, 15), (0, 64, 14)])
def test_restatement_accuracy_vs_dot2(oracle_mod, phi, smax, n_fp64):
    """At the modulus count the form uses for FP64 accuracy, the restatement's componentwise error
    against the compensated reference is no worse than the reference loop's own (FP64 dot products in
    k order); two moduli fewer than needed at phi = 0 is worse than that."""
    M, N, K = 40, 96, 2048
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=3, smax=smax)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
    e_naive = oracle_mod.componentwise_error(oracle_mod.dgemm_naive(A, B, C0, 1.5, 0.5), Cref, den)[0]
    C = oracle_mod.crt_dgemm(A, B, C0, 1.5, 0.5, n_fp64)
    assert oracle_mod.componentwise_error(C, Cref, den)[0] <= e_naive
    if phi == 0 and smax == 0:
        C = oracle_mod.crt_dgemm(A, B, C0, 1.5, 0.5, 12)
        assert oracle_mod.componentwise_error(C, Cref, den)[0] > e_naive


def test_restatement_nonfinite_and_zero_rows(oracle_mod):
    A, B, C0 = oracle_mod.make_problem(6, 5, 40, seed=9)
    A[1, 3] = np.nan
    A[2, :] = 0.0
    B[7, 4] = np.inf
    C = oracle_mod.crt_dgemm(A, B, C0, 2.0, 0.25, 15)
    assert np.all(np.isnan(C[1])) and np.all(np.isnan(C[:, 4]))
    assert np.array_equal(C[2, :4], 0.25 * C0[2, :4])
    good = np.ones(C.shape, bool)
    good[1] = False
    good[:, 4] = False
    assert np.all(np.isfinite(C[good]))


def test_split_residues_are_congruent(oracle_mod):
    A, B, _ = oracle_mod.make_problem(5, 7, 33, phi=20, seed=4)
    n = 16
    sa, sb, ra, rb = oracle_mod.crt_split(A, B, n)
    for i in range(5):
        for k in range(33):
            v = int(np.trunc(np.ldexp(A[i, k], int(sa[i]))))
            for l, m in enumerate(oracle_mod.CRT_MODULI[:n]):
                assert int(ra[l, i, k]) == _sym(v, m)
    for j in range(7):
        for k in range(33):
            v = int(np.trunc(np.ldexp(B[k, j], int(sb[j]))))
            for l, m in enumerate(oracle_mod.CRT_MODULI[:n]):
                assert int(rb[l, j, k]) == _sym(v, m)
