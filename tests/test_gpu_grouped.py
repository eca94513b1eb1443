"""GPU parity of the grouped/batched DGEMM plans (one persistent launch for many uneven problems).

Each problem keeps the reference's contract (routines/dgemm/dgemm.h:9). FP64 form: componentwise
error within (K + 4) u against the compensated oracle. Ozaki form: bit-identical to the CPU
restatement problem by problem. CUDA-graph replay must reproduce the direct launch bit for bit.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import fp64_bound, to_dev

pytestmark = pytest.mark.gpu


def make_set(oracle_mod, count, lo, hi, seed):
    rng = np.random.default_rng(seed)
    dims = np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=(count, 3)))).astype(int)
    probs = []
    for i, (M, N, K) in enumerate(dims):
        A, B, C0 = oracle_mod.make_problem(int(M), int(N), int(K), phi=2, seed=seed * 1000 + i)
        probs.append((A, B, C0, 1.5 if i % 2 else 1.0, 0.5 if i % 3 else 0.0))
    return probs


def upload(torch, probs):
    import libthom_b200 as lt

    dev = []
    table = (lt.GemmProblem * len(probs))()
    for i, (A, B, C0, alpha, beta) in enumerate(probs):
        dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
        dev.append((dA, dB, dC))
        table[i] = lt.GemmProblem(A.shape[0], B.shape[1], A.shape[1], dA.data_ptr(), dB.data_ptr(), dC.data_ptr(),
                                  alpha, beta)
    return dev, table


def plan_run(torch, table, n, form, slices, graph=False, tune=False):
    import libthom_b200 as lt

    L = lt.lib()
    plan = ctypes.c_void_p()
    lt.check(L.lt_grouped_plan_create(table, n, form, slices, ctypes.byref(plan)))
    try:
        if tune:
            ms = ctypes.c_float()
            lt.check(L.lt_grouped_plan_tune(plan, 3, ctypes.byref(ms)))
        if graph:
            lt.check(L.lt_grouped_plan_run_graph(plan, None))
        else:
            lt.check(L.lt_grouped_plan_run(plan, None))
        torch.cuda.synchronize()
        lt.device_status()
        tiles = ctypes.c_int64()
        flops = ctypes.c_double()
        lt.check(L.lt_grouped_plan_info(plan, ctypes.byref(tiles), ctypes.byref(flops)))
        return tiles.value, flops.value
    finally:
        L.lt_grouped_plan_destroy(plan)


@pytest.mark.parametrize("graph,tune", [(False, False), (True, False), (False, True)])
def test_grouped_fp64(cuda, oracle_mod, graph, tune):
    import libthom_b200 as lt

    probs = make_set(oracle_mod, 24, 8, 300, seed=5)
    dev, table = upload(cuda, probs)
    _, flops = plan_run(cuda, table, len(probs), lt.LT_FORM_FP64, 0, graph=graph, tune=tune)
    assert flops == pytest.approx(sum(2.0 * A.shape[0] * A.shape[1] * B.shape[1] for A, B, *_ in probs))
    for (A, B, C0, alpha, beta), (_, _, dC) in zip(probs, dev):
        Cref, den = oracle_mod.dot2_rows(A, B, C0, alpha, beta)
        err = oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)
        assert err[0] <= fp64_bound(A.shape[1]), (A.shape, B.shape, err)


@pytest.mark.parametrize("graph", [False, True])
def test_grouped_fp64_two_size_classes(cuda, oracle_mod, graph):
    """A plan whose big problems (min(M, N) >= 64) run on 64x64 tiles and the rest on 32x32 tiles,
    as two persistent launches (and one captured graph)."""
    import libthom_b200 as lt

    L = lt.lib()
    names = [L.lt_grouped_config_name(i).decode() for i in range(L.lt_grouped_num_configs())]
    big, small = names.index("grouped_cpa_64x64_s3"), names.index("grouped_cpa_32x32_s3")
    probs = make_set(oracle_mod, 20, 8, 300, seed=9)
    dev, table = upload(cuda, probs)
    plan = ctypes.c_void_p()
    lt.check(L.lt_grouped_plan_create(table, len(probs), lt.LT_FORM_FP64, 0, ctypes.byref(plan)))
    try:
        lt.check(L.lt_grouped_plan_set_fp64(plan, big, small, 64))
        name = ctypes.create_string_buffer(128)
        lt.check(L.lt_grouped_plan_config(plan, name, 128))
        assert b">= 64" in name.value, name.value
        if graph:
            lt.check(L.lt_grouped_plan_run_graph(plan, None))
        else:
            lt.check(L.lt_grouped_plan_run(plan, None))
        cuda.cuda.synchronize()
        lt.device_status()
        with pytest.raises(lt.LtError):
            lt.check(L.lt_grouped_plan_set_fp64(plan, big, small, 0))
    finally:
        L.lt_grouped_plan_destroy(plan)
    assert any(min(A.shape[0], B.shape[1]) >= 64 for A, B, *_ in probs)
    assert any(min(A.shape[0], B.shape[1]) < 64 for A, B, *_ in probs)
    for (A, B, C0, alpha, beta), (_, _, dC) in zip(probs, dev):
        Cref, den = oracle_mod.dot2_rows(A, B, C0, alpha, beta)
        err = oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)
        assert err[0] <= fp64_bound(A.shape[1]), (A.shape, B.shape, err)


def upload_offset(torch, probs, offset):
    """`upload` with every matrix starting `offset` doubles into its own allocation (offset 1: the
    base is 8- but not 16-byte aligned)."""
    import libthom_b200 as lt

    def place(a):
        buf = torch.zeros(a.size + offset, dtype=torch.float64, device="cuda")
        view = buf[offset:]
        view.copy_(torch.from_numpy(np.ascontiguousarray(a).ravel()))
        return view.view(a.shape)

    dev = []
    table = (lt.GemmProblem * len(probs))()
    for i, (A, B, C0, alpha, beta) in enumerate(probs):
        dA, dB, dC = place(A), place(B), place(C0)
        dev.append((dA, dB, dC))
        ptr = lambda t: t.data_ptr() if t.numel() else None
        table[i] = lt.GemmProblem(A.shape[0], B.shape[1], A.shape[1], ptr(dA), ptr(dB), ptr(dC), alpha, beta)
    return dev, table


@pytest.mark.parametrize("offset", [0, 1])
def test_grouped_fp64_every_config(cuda, oracle_mod, offset):
    """Every grouped tile configuration (cp.async and TMA staging) on odd and even K and N, bases
    that are not 16-byte aligned (offset 1), M below the tile height and K = 0. The TMA
    configurations copy the operands that no tensor map can describe (odd pitch or base) into even
    pitches on every run: after the first graph replay A is doubled in place and the second replay
    must follow the new values."""
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    shapes = [(5, 7, 9), (64, 64, 64), (130, 66, 33), (97, 128, 200), (33, 31, 0), (200, 3, 150), (1, 1, 1),
              (128, 64, 17), (70, 90, 48)]
    probs = []
    for i, (M, N, K) in enumerate(shapes):
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=2, seed=4000 + i)
        probs.append((A, B, C0, 1.5 if i % 2 else 1.0, 0.5 if i % 3 else 0.0))
    names = [L.lt_grouped_config_name(i).decode() for i in range(L.lt_grouped_num_configs())]
    assert any("tma" in n for n in names) and any("cpa" in n for n in names)
    for cfg, cname in enumerate(names):
        dev, table = upload_offset(torch, probs, offset)
        plan = ctypes.c_void_p()
        lt.check(L.lt_grouped_plan_create(table, len(probs), lt.LT_FORM_FP64, 0, ctypes.byref(plan)))
        try:
            lt.check(L.lt_grouped_plan_set_fp64(plan, cfg, -1, 0))
            lt.check(L.lt_grouped_plan_run_graph(plan, None))
            torch.cuda.synchronize()
            lt.device_status()
            for (A, B, C0, alpha, beta), (_, _, dC) in zip(probs, dev):
                Cref, den = oracle_mod.dot2_rows(A, B, C0, alpha, beta)
                err = oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)
                assert err[0] <= fp64_bound(A.shape[1]), (cname, A.shape, B.shape, err)
            for (A, B, C0, alpha, beta), (dA, _, dC) in zip(probs, dev):
                dA.mul_(2.0)
                dC.copy_(torch.from_numpy(C0))
            lt.check(L.lt_grouped_plan_run_graph(plan, None))
            torch.cuda.synchronize()
            lt.device_status()
            for (A, B, C0, alpha, beta), (_, _, dC) in zip(probs, dev):
                Cref, den = oracle_mod.dot2_rows(2.0 * A, B, C0, alpha, beta)
                err = oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)
                assert err[0] <= fp64_bound(A.shape[1]), (cname, "after A changed", A.shape, B.shape, err)
        finally:
            L.lt_grouped_plan_destroy(plan)


@pytest.mark.parametrize("graph", [False, True])
def test_grouped_ozaki_bit_exact(cuda, oracle_mod, graph):
    import libthom_b200 as lt

    probs = make_set(oracle_mod, 16, 16, 300, seed=9)
    dev, table = upload(cuda, probs)
    plan_run(cuda, table, len(probs), lt.LT_FORM_OZAKI, 7, graph=graph)
    for (A, B, C0, alpha, beta), (_, _, dC) in zip(probs, dev):
        R = oracle_mod.ozaki_dgemm(A, B, C0, alpha, beta, 7)
        assert np.array_equal(dC.cpu().numpy(), R), (A.shape, B.shape)


def test_graph_replay_matches_direct(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    probs = make_set(oracle_mod, 12, 32, 200, seed=3)
    for form, s in ((lt.LT_FORM_FP64, 0), (lt.LT_FORM_OZAKI, 8)):
        dev, table = upload(torch, [(A, B, C0, 1.0, 0.0) for A, B, C0, *_ in probs])
        plan = ctypes.c_void_p()
        lt.check(L.lt_grouped_plan_create(table, len(probs), form, s, ctypes.byref(plan)))
        lt.check(L.lt_grouped_plan_run(plan, None))
        torch.cuda.synchronize()
        first = [d[2].clone() for d in dev]
        for _ in range(3):
            lt.check(L.lt_grouped_plan_run_graph(plan, None))
        torch.cuda.synchronize()
        L.lt_grouped_plan_destroy(plan)
        for a, (_, _, c) in zip(first, dev):
            assert torch.equal(a, c)


def test_grouped_rejects_bad_problems(cuda):
    import libthom_b200 as lt

    L = lt.lib()
    table = (lt.GemmProblem * 1)()
    table[0] = lt.GemmProblem(4, 4, 4, None, None, None, 1.0, 0.0)
    plan = ctypes.c_void_p()
    assert L.lt_grouped_plan_create(table, 1, lt.LT_FORM_FP64, 0, ctypes.byref(plan)) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_grouped_plan_create(table, 0, lt.LT_FORM_FP64, 0, ctypes.byref(plan)) == lt.LT_ERR_INVALID_ARGUMENT


def test_grouped_fp64_at_the_configuration_size(cuda):
    """The batched configuration itself: 512 problems with M, N, K log-uniform in [32, 1024] and
    entries U[-1, 1) (generated on the device), alpha = 1, beta = 0, in one plan run directly and as a
    CUDA graph. Every problem's componentwise error against cuBLAS FP64 (torch.matmul on the same
    device buffers) is within the FP64 bound of its K and the largest within 64 u, and the graph replay
    is bit-identical to the direct run."""
    import libthom_b200 as lt

    torch = cuda
    rng = np.random.default_rng(20260)
    dims = np.rint(np.exp(rng.uniform(np.log(32), np.log(1024), size=(512, 3)))).astype(int)
    bufs = []
    table = (lt.GemmProblem * len(dims))()
    for i, (M, N, K) in enumerate(dims):
        M, N, K = int(M), int(N), int(K)
        A = torch.empty(M, K, dtype=torch.float64, device="cuda")
        B = torch.empty(K, N, dtype=torch.float64, device="cuda")
        C = torch.zeros(M, N, dtype=torch.float64, device="cuda")
        lt.fill(A, M * K, 777 + i, 1, 0)
        lt.fill(B, K * N, 777 + i, 2, 0)
        bufs.append((A, B, C))
        table[i] = lt.GemmProblem(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), 1.0, 0.0)
    plan_run(torch, table, len(dims), lt.LT_FORM_FP64, 0)
    direct = [C.clone() for _, _, C in bufs]
    for _, _, C in bufs:
        C.zero_()
    plan_run(torch, table, len(dims), lt.LT_FORM_FP64, 0, graph=True)
    worst = 0.0
    for (A, B, C), D, (M, N, K) in zip(bufs, direct, dims):
        assert torch.equal(C, D)
        ref = torch.matmul(A, B)
        den = torch.matmul(A.abs(), B.abs())
        err = float(((C - ref).abs() / den.clamp_min(1e-300)).max())
        worst = max(worst, err)
        assert err <= fp64_bound(int(K)), (M, N, K, err)
    # statistical bar, far below the worst case (K + 4) u: both sides round their partial sums, and on
    # this set the largest difference is about 1e-15 (64 u = 7.1e-15)
    assert worst <= 64 * 2.0 ** -53, worst
