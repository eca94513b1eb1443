"""CPU tests of the oracle: pinned against the reference's own host loop and its golden fixtures.

Reference: routines/dgemm/dgemm.cpp:122-133 (getReferenceResults) and the cuRAND-free generator
that replaces dgemm.cpp:100-119.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import ROOT, U, fp64_bound


def _cases(golden):
    for i in range(int(golden["ncases"][0])):
        M, N, K, phi, smax, seed = (int(x) for x in golden[f"case{i}_params"])
        alpha, beta = (float(x) for x in golden[f"case{i}_scalars"])
        yield i, M, N, K, phi, smax, seed, alpha, beta


def test_generator_pinned(oracle_mod, golden):
    gen = [oracle_mod.fill(1, 16, st, phi, 1234)[0] for st in (1, 2, 3) for phi in (0, 8)]
    assert np.array_equal(np.stack(gen), golden["generator_first16"])


def test_generator_ranges(oracle_mod):
    x = oracle_mod.fill(256, 256, 1, 0)
    assert x.min() >= -1.0 and x.max() < 1.0
    assert abs(x.mean()) < 0.01
    y = oracle_mod.fill(256, 256, 1, 8)
    e = np.frexp(y[y != 0])[1]
    assert e.min() >= -8 - 52 and e.max() <= 9
    # same stream and seed -> same values; different stream -> different values
    assert np.array_equal(oracle_mod.fill(3, 5, 7, 2), oracle_mod.fill(3, 5, 7, 2))
    assert not np.array_equal(oracle_mod.fill(3, 5, 7, 2), oracle_mod.fill(3, 5, 8, 2))


def test_row_col_scaling(oracle_mod):
    A = oracle_mod.fill(20, 30, 1, 0)
    S = A.copy()
    oracle_mod.scale_rows(S, 1234, 4, 64)
    ratio = S / A
    r = np.log2(np.abs(ratio[:, 0]))
    assert np.all(r == np.round(r)) and np.abs(r).max() <= 64
    assert np.all(ratio == ratio[:, :1])  # one power of two per row


def test_naive_matches_golden_bit_exact(oracle_mod, golden):
    for i, M, N, K, phi, smax, seed, alpha, beta in _cases(golden):
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=seed, smax=smax)
        d = hashlib.sha256()
        for a in (A, B, C0):
            d.update(np.ascontiguousarray(a).tobytes())
        assert bytes(golden[f"case{i}_digest"]).decode() == d.hexdigest(), f"case {i}: inputs differ"
        C = oracle_mod.dgemm_naive(A, B, C0, alpha, beta)
        assert np.array_equal(C, golden[f"case{i}_C"]), f"case {i}"


def test_naive_matches_reference_build(oracle_mod):
    if oracle_mod.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    for (M, N, K) in [(37, 41, 53), (1, 1, 1), (70, 3, 129)]:
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=4, seed=99)
        assert np.array_equal(oracle_mod.dgemm_naive(A, B, C0, 0.75, -1.25),
                              oracle_mod.dgemm_ref(A, B, C0, 0.75, -1.25))


@pytest.mark.parametrize("M,N,K", [(64, 64, 64), (17, 23, 31), (100, 130, 257), (5, 300, 7)])
def test_blocked_within_fp64_bound(oracle_mod, M, N, K):
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=8, seed=5)
    Cb = oracle_mod.dgemm_blocked(A, B, C0, 1.5, 0.5)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
    err = oracle_mod.componentwise_error(Cb, Cref, den)
    assert err[0] <= fp64_bound(K), err
    assert err[3] == 0


def test_dot2_is_more_accurate_than_naive(oracle_mod):
    M, N, K = 40, 40, 2000
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=16, seed=3)
    Cn = oracle_mod.dgemm_naive(A, B, C0, 1.0, 0.0)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 0.0)
    err = oracle_mod.componentwise_error(Cn, Cref, den)
    assert 0 < err[0] <= fp64_bound(K)
    # Dot2 of a subset equals Dot2 of the full set
    Cs, dens = oracle_mod.dot2_rows(A, B, C0, 1.0, 0.0, rows=np.array([3, 17, 39]))
    assert np.array_equal(Cs, Cref[[3, 17, 39]]) and np.array_equal(dens, den[[3, 17, 39]])


def test_ozaki_slices_reconstruct(oracle_mod):
    """Slices are the balanced base-256 digits of trunc(a 2^(8s-2-sigma)): the top digit in
    [-64, 64], the others in [-128, 127], a = 2^(sigma+2) sum_p q_p 256^-p up to a truncation
    toward zero smaller than 2^(sigma-(8s-2))."""
    from fractions import Fraction

    A, B, _ = oracle_mod.make_problem(30, 20, 50, phi=20, seed=11)
    for s in (1, 4, 8, 12):
        sigma, tau, sa, sb = oracle_mod.ozaki_split(A, B, s)
        for sl in (sa, sb):
            assert np.abs(sl[0].astype(np.int64)).max() <= 64
            assert sl.min() >= -128 and sl.max() <= 127
        assert np.all(sa[:, :, 50:] == 0)  # K padding
        for (i, k) in [(0, 0), (3, 17), (29, 49), (11, 5)]:
            V = sum(int(sa[p, i, k]) * 256 ** (s - 1 - p) for p in range(s))  # exact integer
            x = Fraction(A[i, k]) * Fraction(2) ** (8 * s - 2 - int(sigma[i]))
            assert abs(V) == int(abs(x)) and (V == 0 or (V > 0) == (x > 0))  # trunc toward zero
        for (k, j) in [(0, 0), (49, 19), (7, 3)]:
            V = sum(int(sb[p, j, k]) * 256 ** (s - 1 - p) for p in range(s))
            x = Fraction(B[k, j]) * Fraction(2) ** (8 * s - 2 - int(tau[j]))
            assert abs(V) == int(abs(x)) and (V == 0 or (V > 0) == (x > 0))


def test_ozaki_restatement_accuracy(oracle_mod):
    M, N, K = 60, 50, 300
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=0, seed=21)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
    errs = []
    for s in range(3, 11):
        C = oracle_mod.ozaki_dgemm(A, B, C0, 1.5, 0.5, s)
        errs.append(oracle_mod.componentwise_error(C, Cref, den)[0])
    assert all(errs[i + 1] <= errs[i] for i in range(len(errs) - 1)), errs
    # each slice buys about 8 bits
    assert errs[0] / errs[4] > 2.0 ** 28
    # eight slices reach FP64 accuracy on unscaled data
    assert errs[5] <= fp64_bound(K)
    assert errs[5] <= 64 * U


def test_ozaki_nan_inf_and_zero_rows(oracle_mod):
    M, N, K = 12, 9, 40
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=8)
    A[3, 7] = np.nan
    B[11, 5] = np.inf
    A[6, :] = 0.0
    C = oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 0.5, 6)
    assert np.all(np.isnan(C[3, :])) and np.all(np.isnan(C[:, 5]))
    rows = [i for i in range(M) if i != 3]
    cols = [j for j in range(N) if j != 5]
    assert np.all(np.isfinite(C[np.ix_(rows, cols)]))
    assert np.array_equal(C[6, cols], 0.5 * C0[6, cols])


def test_ozaki_long_k_groups(oracle_mod):
    """K beyond the INT32-safe group length splits the band into several groups; the result is
    still accurate (no INT32 overflow)."""
    M, N, K = 4, 3, 40000
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=13)
    A[:] = np.where(A >= 0, 1.0 - 2.0 ** -40, -(1.0 - 2.0 ** -40))  # digits near their extremes
    B[:] = np.abs(A[0, :])[:, None]
    C = oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 0.0, 8)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 0.0)
    assert oracle_mod.componentwise_error(C, Cref, den)[0] < 1e-13


def test_analytic_slices_monotone(oracle_mod):
    a = [oracle_mod.analytic_slices(t, 0) for t in (1e-6, 1e-10, 1e-12, 1e-14, 1e-15)]
    assert a == sorted(a) and a[-1] >= 8
    assert oracle_mod.analytic_slices(1e-12, 64) > oracle_mod.analytic_slices(1e-12, 0)


@pytest.mark.parametrize("phi,smax", [(0, 0), (8, 0), (32, 0), (0, 64)])
def test_analytic_count_is_conservative(oracle_mod, phi, smax):
    """The analytic count meets its tolerance on every sampled problem (it is the fallback)."""
    M, N, K = 40, 30, 256
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=phi + smax, smax=smax)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 0.0)
    g = oracle_mod.gap_bits(A, B)
    for tol in (1e-12, 1e-14):
        s = oracle_mod.analytic_slices(tol, g)
        if s == 12 and (s + 3) * 2.0 ** (g + 2 - 7 * s) > tol:
            continue  # beyond the largest slice count: no claim
        C = oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 0.0, s)
        assert oracle_mod.componentwise_error(C, Cref, den)[0] <= tol, (phi, smax, tol, s, g)


def test_mlp_backward_matches_finite_differences(oracle_mod):
    rng = np.random.default_rng(0)
    P = oracle_mod.SEL_P
    params = (rng.standard_normal(P) * 0.2).astype(np.float32)
    x = rng.random((6, oracle_mod.SEL_F)).astype(np.float32)
    y = rng.integers(0, 8, 6).astype(np.int32)
    loss, g = oracle_mod.mlp_backward(params, x, y)
    for i in rng.choice(P, 25, replace=False):
        h = 1e-2
        pp = params.astype(np.float64)
        for sign, store in ((1, "p"), (-1, "m")):
            q = pp.copy()
            q[i] += sign * h
            val = oracle_mod.mlp_backward(q.astype(np.float32), x, y)[0]
            if store == "p":
                lp = val
            else:
                lm = val
        # the float32 parameter perturbation is exact for h = 1e-2 only up to float rounding
        hp = float(np.float32(pp[i] + h)) - pp[i]
        hm = pp[i] - float(np.float32(pp[i] - h))
        fd = (lp - lm) / (hp + hm)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])), (i, fd, g[i])
    probs = oracle_mod.mlp_forward(params, x)
    assert np.allclose(probs.sum(axis=1), 1.0, atol=1e-6)


# ---- FP16 HGEMM host check (routines/hgemm/hgemm.cu:135-149) -------------------------------------
def test_half_conversions_exhaustive(oracle_mod):
    """FP16 -> float over all 65536 patterns and float -> FP16 (ties to even, subnormals, overflow)
    on every midpoint between neighbouring FP16 values, against numpy's IEEE conversions."""
    L = oracle_mod.lib()
    allh = np.arange(65536, dtype=np.uint16)
    ref = allh.view(np.float16).astype(np.float32)
    got = np.array([L.oracle_half_to_float(int(h)) for h in allh], dtype=np.float32)
    fin = np.isfinite(ref)
    assert np.array_equal(ref[fin].view(np.uint32), got[fin].view(np.uint32))
    assert np.all(np.isnan(got[np.isnan(ref)]))
    pos = np.arange(0x7c00, dtype=np.uint16).view(np.float16).astype(np.float64)
    mids = ((pos[:-1] + pos[1:]) / 2).astype(np.float32)  # exact in float32
    xs = np.concatenate([mids, -mids, np.float32([65519.0, 65520.0, 1e9, 2.0 ** -26, 2.0 ** -25, 0.0])])
    with np.errstate(over="ignore"):
        want = xs.astype(np.float16).view(np.uint16)
    got = np.array([L.oracle_float_to_half(float(x)) for x in xs], dtype=np.uint16)
    assert np.array_equal(want, got)


def test_hgemm_ref_matches_golden_bit_exact(oracle_mod):
    """The restated HGEMM check against the fixtures made by the reference's own compiled loop."""
    g = np.load(ROOT / "tests" / "golden" / "hgemm_ref.npz")
    for i in range(int(g["ncases"][0])):
        alpha, beta = (float(x) for x in g[f"case{i}_scalars"])
        C = oracle_mod.hgemm_ref(g[f"case{i}_A"], g[f"case{i}_B"], g[f"case{i}_C0"], alpha, beta)
        assert np.array_equal(C, g[f"case{i}_C"]), i
    # and a subset of rows gives the same rows
    A, B, C0 = g["case2_A"], g["case2_B"], g["case2_C0"]
    rows = np.array([0, 5, 23])
    assert np.array_equal(oracle_mod.hgemm_ref(A, B, C0, 1.0, 0.0, rows=rows), g["case2_C"][rows])


def test_hgemm_ref_matches_reference_build(oracle_mod):
    """Where the reference sources are present: a fresh case through both loops, bit for bit."""
    A, B, C0 = oracle_mod.make_half_problem(33, 47, 129, seed=99, lo=-3.0, hi=3.0)
    ref = oracle_mod.hgemm_ref_loop(A, B, C0, int(oracle_mod.half_bits(-0.75)), int(oracle_mod.half_bits(2.0)))
    if ref is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")
    assert np.array_equal(oracle_mod.hgemm_ref(A, B, C0, -0.75, 2.0), ref)


def test_hgemm_exact_rows_bounds_the_float_loop(oracle_mod):
    """The float64 value and denominator used for GPU tolerances: the reference's float loop lies
    within K u32 den + half an FP16 ulp of it."""
    A, B, C0 = oracle_mod.make_half_problem(20, 30, 700, seed=3, lo=-1.0, hi=1.0)
    C = oracle_mod.hgemm_ref(A, B, C0, 1.5, 0.5).view(np.float16).astype(np.float64)
    ex, den = oracle_mod.hgemm_exact_rows(A, B, C0, 1.5, 0.5)
    tol = (700 + 4) * 2.0 ** -24 * den + 2.0 ** -11 * np.abs(ex) + 2.0 ** -25
    assert np.all(np.abs(C - ex) <= tol)
