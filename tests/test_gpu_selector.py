"""GPU checks of the learned slice-count selector: features and MLP kernels against the CPU oracle
(gradient check included), training progress, the analytic fallback, and what the trained network
gains over the analytic count on held-out problems.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu
WEIGHTS = Path(__file__).resolve().parents[1] / "libthom_b200" / "selector_weights.bin"


def gpu_features(torch, A, B, tol):
    import libthom_b200 as lt

    dA, dB = to_dev(torch, A), to_dev(torch, B)
    f = torch.empty(lt.LT_SEL_FEATURES, dtype=torch.float32, device="cuda")
    lt.check(lt.lib().lt_ozaki_features(dA.data_ptr(), dB.data_ptr(), A.shape[0], B.shape[1], A.shape[1], tol,
                                        f.data_ptr(), None))
    return f.cpu().numpy()


@pytest.mark.parametrize("M,N,K,phi,smax", [(300, 200, 150, 0, 0), (90, 17, 500, 30, 40), (1, 1, 1, 0, 0)])
def test_features_match_oracle(cuda, oracle_mod, M, N, K, phi, smax):
    A, B, _ = oracle_mod.make_problem(M, N, K, phi=phi, seed=M + N, smax=smax)
    A[0, 0] = 0.0
    f = gpu_features(cuda, A, B, 1e-14)
    r = oracle_mod.features(A, B, 1e-14)
    assert np.array_equal(f, r), np.abs(f - r).max()


def rand_params(seed, scale=0.3):
    import libthom_b200 as lt

    return (np.random.default_rng(seed).standard_normal(lt.LT_SEL_PARAMS) * scale).astype(np.float32)


def test_mlp_forward_matches_oracle(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    p = rand_params(1)
    x = np.random.default_rng(2).random((64, lt.LT_SEL_FEATURES)).astype(np.float32)
    out = torch.empty(64, lt.LT_SEL_CLASSES, dtype=torch.float32, device="cuda")
    dp, dx = to_dev(torch, p), to_dev(torch, x)  # keep the buffers alive across the launch
    lt.check(lt.lib().lt_mlp_forward(dp.data_ptr(), dx.data_ptr(), 64, out.data_ptr(), None))
    assert np.allclose(out.cpu().numpy(), oracle_mod.mlp_forward(p, x), atol=2e-6)


def test_mlp_gradient_check(cuda, oracle_mod):
    """Backward kernel (per-sample gradients, fixed-order batch mean) vs the double-precision CPU
    oracle, which is itself checked against finite differences in test_oracle.py."""
    import libthom_b200 as lt

    torch = cuda
    p = rand_params(3)
    rng = np.random.default_rng(4)
    x = rng.random((96, lt.LT_SEL_FEATURES)).astype(np.float32)
    y = rng.integers(0, lt.LT_SEL_CLASSES, 96).astype(np.int32)
    g = torch.empty(lt.LT_SEL_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    dp, dx, dy = to_dev(torch, p), to_dev(torch, x), to_dev(torch, y)
    lt.check(lt.lib().lt_mlp_backward(dp.data_ptr(), dx.data_ptr(), dy.data_ptr(), 96, g.data_ptr(),
                                      loss.data_ptr(), None))
    ref_loss, ref_g = oracle_mod.mlp_backward(p, x, y)
    gg = g.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - ref_loss) <= 1e-5 * max(1.0, abs(ref_loss))
    assert np.all(np.abs(gg - ref_g) <= 2e-6 + 1e-4 * np.abs(ref_g)), np.abs(gg - ref_g).max()


def test_training_reduces_loss(cuda):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    rng = np.random.default_rng(5)
    x = rng.random((256, lt.LT_SEL_FEATURES)).astype(np.float32)
    y = (x[:, 0] * 7.99).astype(np.int32)  # a learnable labelling
    p = to_dev(torch, rand_params(6, 0.1))
    m, v, g = (torch.zeros_like(p) for _ in range(3))
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    xd, yd = to_dev(torch, x), to_dev(torch, y)
    losses = []
    for step in range(1, 301):
        lt.check(L.lt_mlp_train_step(p.data_ptr(), m.data_ptr(), v.data_ptr(), g.data_ptr(), xd.data_ptr(),
                                     yd.data_ptr(), 256, 3e-3, step, loss.data_ptr(), None))
        losses.append(float(loss.item()))
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])


def select(torch, A, B, tol):
    import libthom_b200 as lt

    dA, dB = to_dev(torch, A), to_dev(torch, B)
    s, learned, gap = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lt.check(lt.lib().lt_ozaki_select_info(dA.data_ptr(), dB.data_ptr(), A.shape[0], B.shape[1], A.shape[1], tol,
                                           ctypes.byref(s), ctypes.byref(learned), ctypes.byref(gap), None))
    return s.value, bool(learned.value), gap.value


def test_analytic_fallback_without_weights(cuda, oracle_mod):
    import libthom_b200 as lt

    L = lt.lib()
    lt.check(L.lt_selector_set_params(None))
    try:
        for phi, smax in ((0, 0), (16, 0), (0, 40)):
            A, B, _ = oracle_mod.make_problem(120, 80, 200, phi=phi, seed=phi + smax, smax=smax)
            s, learned, gap = select(cuda, A, B, 1e-14)
            assert not learned
            assert gap == oracle_mod.gap_bits(A, B)
            assert s == oracle_mod.analytic_slices(1e-14, gap)
    finally:
        if WEIGHTS.exists():
            w = np.fromfile(WEIGHTS, dtype=np.float32)
            lt.check(L.lt_selector_set_params(w.ctypes.data))


def test_trained_selector_gains_over_analytic(cuda, oracle_mod):
    """Held-out problems (seeds never used in training): with the trained weights the selector
    picks fewer slices than the analytic count on average and misses the tolerance (checked against
    the compensated oracle, not the FP64 result the labels came from) on no more of the problems where
    it is reachable than the analytic count does. A problem is unreachable when
    even the largest slice count misses the tolerance (wide exponent spread in both operands): no
    choice of s can meet it, so it does not count as a miss of the selector."""
    import libthom_b200 as lt

    if not WEIGHTS.exists():
        pytest.fail("libthom_b200/selector_weights.bin missing: run python -m libthom_b200.selector_train")
    L = lt.lib()
    w = np.fromfile(WEIGHTS, dtype=np.float32)
    lt.check(L.lt_selector_set_params(w.ctypes.data))
    torch = cuda
    rng = np.random.default_rng(424242)
    saved, misses, misses_analytic, n = [], 0, 0, 0

    def error_at(dA, dB, M, N, K, s, Cref, den):
        dC = torch.zeros(M, N, dtype=torch.float64, device="cuda")
        lt.dgemm_ozaki(dA, dB, dC, M, N, K, 1.0, 0.0, slices=s)
        return oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)[0]

    for i in range(24):
        M, N, K = (int(rng.integers(64, 257)) for _ in range(3))
        phi = int(rng.integers(0, 65))
        smax = int(rng.integers(0, 65)) if i % 2 else 0
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=10**9 + i, smax=smax)
        Cref, den = oracle_mod.dot2_rows(A, B, None, 1.0, 0.0)
        tol = (1e-12, 1e-14, 1e-15)[i % 3]
        s, learned, _ = select(torch, A, B, tol)
        dA, dB = to_dev(torch, A), to_dev(torch, B)
        gap = ctypes.c_int()
        lt.check(L.lt_ozaki_gap_bits(dA.data_ptr(), dB.data_ptr(), M, N, K, ctypes.byref(gap), None))
        assert gap.value == oracle_mod.gap_bits(A, B)
        sa = oracle_mod.analytic_slices(tol, gap.value)
        if not learned:
            assert s == sa
        saved.append(sa - s)
        if error_at(dA, dB, M, N, K, lt.LT_OZAKI_MAX_SLICES, Cref, den) > tol:
            continue  # unreachable
        misses += error_at(dA, dB, M, N, K, s, Cref, den) > tol
        misses_analytic += error_at(dA, dB, M, N, K, sa, Cref, den) > tol
        n += 1
    assert np.mean(saved) >= 1.0, saved
    assert n >= 8, n
    assert misses <= misses_analytic, (misses, misses_analytic, n)


def test_ozaki_auto_meets_tolerance(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    M, N, K = 256, 192, 512
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=4, seed=77)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
    L.lt_set_ozaki_tolerance(1e-12)
    try:
        dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
        ms = lt.dgemm("ozaki_auto", dA, dB, dC, M, N, K, 1.5, 0.5)
        assert ms > 0
        assert oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)[0] <= 1e-12
    finally:
        L.lt_set_ozaki_tolerance(1e-15)


def _install_weights(lt, on):
    L = lt.lib()
    if on:
        w = np.fromfile(WEIGHTS, dtype=np.float32)
        lt.check(L.lt_selector_set_params(w.ctypes.data))
    else:
        lt.check(L.lt_selector_set_params(None))


@pytest.mark.parametrize("weights", [True, False])
def test_auto_plan_chooses_on_the_device_what_the_host_path_chooses(cuda, oracle_mod, weights):
    """lt_ozaki_auto_plan: its graph picks the slice count on the device with the same rule and kernels
    as lt_ozaki_select_info (learned when the network is confident, else the analytic count from the
    exponent gaps; without weights always the analytic count), and its result is lt_dgemm_ozaki's with
    that count, bit for bit. A replay after the data behind the pointers changed chooses again."""
    import libthom_b200 as lt

    if weights and not WEIGHTS.exists():
        pytest.fail("libthom_b200/selector_weights.bin missing")
    torch = cuda
    _install_weights(lt, weights)
    try:
        cases = [(300, 200, 150, 0, 0, 1e-12), (256, 320, 700, 8, 0, 1e-14), (90, 17, 500, 30, 40, 1e-15),
                 (513, 260, 1000, 2, 20, 1e-12)]
        for M, N, K, phi, smax, tol in cases:
            A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=M + K, smax=smax)
            dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
            plan = lt.OzakiAutoPlan(dA, dB, dC, M, N, K, 1.5, 0.5, tol)
            try:
                for rep in range(2):
                    if rep == 1:  # new data behind the same pointers
                        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=(phi + 17) % 40, seed=M + K + 1, smax=smax)
                        dA.copy_(torch.from_numpy(A))
                        dB.copy_(torch.from_numpy(B))
                    dC.copy_(torch.from_numpy(C0))
                    plan.run()
                    torch.cuda.synchronize()
                    lt.device_status()
                    s, learned = plan.choice()
                    hs, hlearned, _ = select(torch, A, B, tol)
                    assert (s, learned) == (hs, hlearned), (M, N, K, rep)
                    if not weights:
                        assert not learned
                    ref = to_dev(torch, C0)
                    lt.dgemm_ozaki(dA, dB, ref, M, N, K, 1.5, 0.5, slices=s)
                    torch.cuda.synchronize()
                    assert np.array_equal(dC.cpu().numpy(), ref.cpu().numpy()), (M, N, K, rep, s)
            finally:
                plan.close()
    finally:
        _install_weights(lt, WEIGHTS.exists())



def test_any_form_plan_picks_native_fp64_where_the_cost_model_does(cuda, oracle_mod):
    """With LT_AUTO_PLAN_ANY_FORM a shape on which native FP64 beats even 3 slices (512^3) becomes a
    plan of the FP64 kernel alone (choice: 0 slices), one where the slice form wins (2048^3) keeps the
    selection; both results are within the FP64 bound against the compensated reference."""
    import libthom_b200 as lt
    from conftest import fp64_bound

    torch = cuda
    _install_weights(lt, WEIGHTS.exists())
    for n, want_fp64 in ((512, True), (2048, False)):
        A = torch.empty(n, n, dtype=torch.float64, device="cuda")
        B = torch.empty_like(A)
        C = torch.zeros_like(A)
        lt.fill(A, n * n, 11, 1, 0)
        lt.fill(B, n * n, 11, 2, 0)
        rows = torch.linspace(0, n - 1, 4, device="cuda").round().to(torch.int64)
        Cref = torch.empty(4, n, dtype=torch.float64, device="cuda")
        den = torch.empty_like(Cref)
        lt.dot2_rows(A, B, C, n, n, n, 1.0, 0.0, rows, Cref, den)
        plan = lt.OzakiAutoPlan(A, B, C, n, n, n, 1.0, 0.0, 1e-12, forms=lt.LT_AUTO_PLAN_ANY_FORM)
        try:
            plan.run()
            torch.cuda.synchronize()
            lt.device_status()
            s, _ = plan.choice()
            assert (s == 0) == want_fp64, (n, s)
            e = lt.componentwise_error(C[rows].contiguous(), Cref, den, Cref.numel())[0]
            assert e <= (fp64_bound(n) if s == 0 else 1e-12), (n, s, e)
        finally:
            plan.close()


def test_auto_plan_beats_the_fixed_slice_count_for_the_tolerance(cuda, oracle_mod):
    """Held-out problems from the selector's own distribution (selector_train.draw_shape: square,
    tall-skinny and long-K shapes up to 2048, exponent spread phi over 0..64, row/column scaling) at
    tolerance 1e-12: 8 drawn as they come and 4 from the distribution's tail (scaled rows and
    columns with phi >= 56), since 1 in 13 of its problems needs 10 or more slices at 1e-12 and a
    fixed count must cover them (12 on 800 held-out problems). The fixed slice count a user without
    the selector would need is the smallest meeting the tolerance on every problem of the set where
    any count does. The plans (LT_AUTO_PLAN_ANY_FORM: the choice inside their graphs, no host round
    trip, native FP64 where the cost model prefers it to the chosen count) run the whole set in less
    time than that fixed count, and meet the tolerance wherever it is reachable (errors on 4 sampled
    rows against the compensated reference on the device)."""
    import libthom_b200 as lt
    from libthom_b200 import selector_train as st

    if not WEIGHTS.exists():
        pytest.fail("libthom_b200/selector_weights.bin missing")
    torch = cuda
    _install_weights(lt, True)
    tol = 1e-12
    rng = np.random.default_rng(55555)
    probs = []
    for i in range(12):
        fam, M, N, K, phi, smax, seed = st.draw_shape(rng)
        while i >= 8 and fam == 0:  # the tail: a scaled family
            fam, M, N, K, phi, smax, seed = st.draw_shape(rng)
        if i >= 8:
            phi, smax = int(rng.integers(56, 65)), int(rng.integers(48, 65))
        A = torch.empty(M, K, dtype=torch.float64, device="cuda")
        B = torch.empty(K, N, dtype=torch.float64, device="cuda")
        lt.fill(A, M * K, seed, 1, phi)
        lt.fill(B, K * N, seed, 2, phi)
        if smax:
            lt.scale_rows(A, M, K, seed, 4, smax)
            lt.scale_cols(B, K, N, seed, 5, smax)
        C = torch.zeros(M, N, dtype=torch.float64, device="cuda")
        rows = torch.linspace(0, M - 1, min(M, 4), device="cuda").round().to(torch.int64)
        Cref = torch.empty(rows.numel(), N, dtype=torch.float64, device="cuda")
        den = torch.empty_like(Cref)
        lt.dot2_rows(A, B, C, M, N, K, 1.0, 0.0, rows, Cref, den)
        probs.append((A, B, C, M, N, K, rows, Cref, den))

    def err(p):
        A, B, C, M, N, K, rows, Cref, den = p
        torch.cuda.synchronize()
        return lt.componentwise_error(C[rows].contiguous(), Cref, den, Cref.numel())[0]

    def run_fixed(p, s):
        lt.dgemm_ozaki(p[0], p[1], p[2], p[3], p[4], p[5], 1.0, 0.0, slices=s)

    reachable = []
    for p in probs:
        run_fixed(p, lt.LT_OZAKI_MAX_SLICES)
        reachable.append(err(p) <= tol)
    fixed = None
    for s in range(3, lt.LT_OZAKI_MAX_SLICES + 1):
        ok = True
        for p, r in zip(probs, reachable):
            if r:
                run_fixed(p, s)
                ok = ok and err(p) <= tol
        if ok:
            fixed = s
            break
    assert fixed is not None and sum(reachable) >= 8, reachable
    plans = [lt.OzakiAutoPlan(p[0], p[1], p[2], p[3], p[4], p[5], 1.0, 0.0, tol, forms=lt.LT_AUTO_PLAN_ANY_FORM)
             for p in probs]
    try:
        for pl, p, r in zip(plans, probs, reachable):
            pl.run()
            if r:
                assert err(p) <= tol, pl.choice()

        def timed(fn, reps=5):
            for _ in range(2):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        t_fixed = timed(lambda: [run_fixed(p, fixed) for p in probs])
        t_plan = timed(lambda: [pl.run() for pl in plans])
        lt.device_status()
        chosen = [pl.choice()[0] for pl in plans]
        assert t_plan < t_fixed, (t_plan, t_fixed, fixed, chosen)
    finally:
        for pl in plans:
            pl.close()
