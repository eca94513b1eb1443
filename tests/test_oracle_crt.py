"""CPU checks of the CRT form (Ozaki scheme II): the moduli, the exactness of the FP64
reconstruction the kernel and the restatement share, the restatement's accuracy against the
compensated Dot2 reference, and that the library derives the same operand bits as the oracle."""
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
    """The limb sums stay below 2^53 and Q = rint(L_hi F_hi + L_lo F_lo) is exact for every integer
    within Mprod / 4 in magnitude (the bound the scaling guarantees); values at the edges included."""
    c = oracle_mod.crt_constants(n, 1024)
    Mp, mods, nl = c["Mprod"], [int(m) for m in c["mods"]], c["nl"]
    rng = random.Random(n)
    xs = [0, 1, -1, Mp // 4 - 1, -(Mp // 4) + 1] + [rng.randrange(-(Mp // 4) + 1, Mp // 4) for _ in range(400)]
    xs += [rng.randrange(-2 ** 40, 2 ** 40) for _ in range(100)]
    for x in xs:
        res = [_sym(x, m) for m in mods]
        L = [0.0] * nl
        for l in range(n):
            for k in range(nl):
                L[k] = float(res[l]) * float(c["P"][l][k]) + L[k]
                assert abs(L[k]) < 2.0 ** 53
        Q = round(L[nl - 1] * c["f_hi"] + L[nl - 2] * c["f_lo"])
        S = sum(r * ((Mp // m) * pow((Mp // m) % m, -1, m)) for r, m in zip(res, mods))
        assert S - Q * Mp == x


def test_operand_bits_respect_the_bound(oracle_mod):
    for n in range(oracle_mod.CRT_MIN, oracle_mod.CRT_MAX + 1):
        for K in (1, 7, 1000, 8192, 65536, 130000, 2 ** 31 - 1):
            c = oracle_mod.crt_constants(n, K)
            assert 4 * K * 2 ** (c["pa"] + c["pb"]) <= c["Mprod"]
            if c["pa"] < 62 and c["pb"] < 62:  # the largest such exponent sum
                assert 4 * K * 2 ** (c["pa"] + c["pb"] + 1) > c["Mprod"]


def test_library_constants_match_the_oracle(oracle_mod):
    import libthom_b200 as lt

    for n in range(oracle_mod.CRT_MIN, oracle_mod.CRT_MAX + 1):
        for K in (1, 33, 8192, 65536, 131072, 2 ** 31 - 1):
            c = oracle_mod.crt_constants(n, K)
            pa, pb, mods = lt.ozaki_crt_info(n, K)
            assert (pa, pb) == (c["pa"], c["pb"]), (n, K)
            assert mods == list(oracle_mod.CRT_MODULI[:n])
    L = lt.lib()
    assert L.lt_ozaki_crt_info(7, 100, None, None, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_crt_info(21, 100, None, None, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(None, None, None, 4, 4, 4, 1.0, 0.0, 15, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(0x1000, 0x1000, 0x1000, 4, 4, 4, 1.0, 0.0, 7, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ozaki_crt(0x1000, 0x1000, 0x1000, 4, 4, 9_000_000, 1.0, 0.0, 15, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_crt_workspace_size(8192, 8192, 8192, 15) > 15 * 3 * 8192 * 8192


@pytest.mark.parametrize("phi,smax,n_fp64", [(0, 0, 15), (8, 0, 15), (32, 0, 16), (0, 64, 15)])
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
        C = oracle_mod.crt_dgemm(A, B, C0, 1.5, 0.5, 13)
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
    c = oracle_mod.crt_constants(n, 33)
    sigma, tau, ra, rb = oracle_mod.crt_split(A, B, n)
    for i in range(5):
        for k in range(33):
            v = int(np.trunc(np.ldexp(A[i, k], c["pa"] - int(sigma[i]))))
            for l, m in enumerate(oracle_mod.CRT_MODULI[:n]):
                assert int(ra[l, i, k]) == _sym(v, m)
