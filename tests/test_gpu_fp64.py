"""GPU parity of the native FP64 tensor-core DGEMM (dgemm_tc100 / lt_dgemm_fp64).

Oracle: the reference's own host loop (golden fixtures from routines/dgemm/dgemm.cpp:122-133) and
the compensated Dot2 oracle. Tolerances, both asserted: the worst-case componentwise bound of an FP64
dot product of length K in any order, (K + 4) u relative to |alpha||A||B| + |beta||C0| (u = 2^-53),
and the statistical bar max(4 e_cublas, 16 u), e_cublas being cuBLAS DGEMM's componentwise error on
the same inputs (a kernel that lost a few bits would fail it; the worst case alone allows thousands
of times the observed error at K = 8192).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import U, fp64_bound, tight_fp64_bound, to_dev

pytestmark = pytest.mark.gpu


def run_fp64(torch, A, B, C0, alpha, beta, config=-1, offset=0):
    import libthom_b200 as lt

    M, K = A.shape
    N = B.shape[1]
    if offset:
        # place each matrix 8 bytes past a 16-byte boundary (forces the cp.async path)
        bufs = []
        for x in (A, B, C0):
            t = torch.empty(x.size + 1, dtype=torch.float64, device="cuda")
            t[1:] = torch.from_numpy(np.ascontiguousarray(x).ravel()).cuda()
            bufs.append(t)
        dA, dB, dC = (t[1:] for t in bufs)
    else:
        dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    lt.dgemm_fp64(dA, dB, dC, M, N, K, alpha, beta, config=config)
    torch.cuda.synchronize()
    lt.device_status()
    return dC.cpu().numpy().reshape(M, N)


def cublas_error(torch, A, B, C0, alpha, beta, Cref, den):
    """cuBLAS DGEMM's componentwise error on the same inputs (the statistical bar's yardstick)."""
    import libthom_b200 as lt

    M, K = A.shape
    N = B.shape[1]
    dC = to_dev(torch, C0)
    lt.dgemm_cublas(to_dev(torch, A), to_dev(torch, B), dC, M, N, K, alpha, beta)
    torch.cuda.synchronize()
    return _cw(dC.cpu().numpy(), Cref, den)


def _cw(C, Cref, den):
    import oracle

    return oracle.componentwise_error(C, Cref, den)[0]


def check(C, Cref, den, K, e_cublas, label=""):
    err = _cw(C, Cref, den)
    assert err <= fp64_bound(K), (label, err)
    assert err <= tight_fp64_bound(e_cublas), (label, err, e_cublas)


def test_golden_cases(cuda, oracle_mod, golden):
    for i in range(int(golden["ncases"][0])):
        M, N, K, phi, smax, seed = (int(x) for x in golden[f"case{i}_params"])
        alpha, beta = (float(x) for x in golden[f"case{i}_scalars"])
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=seed, smax=smax)
        C = run_fp64(cuda, A, B, C0, alpha, beta)
        Cref, den = oracle_mod.dot2_rows(A, B, C0, alpha, beta)
        check(C, Cref, den, K, cublas_error(cuda, A, B, C0, alpha, beta, Cref, den), i)
        # and against the reference loop's own output (both FP64: same bound, twice)
        err_ref = oracle_mod.componentwise_error(C, golden[f"case{i}_C"], den)
        assert err_ref[0] <= 2 * fp64_bound(K), (i, err_ref)


def test_every_config(cuda, oracle_mod):
    import libthom_b200 as lt

    names = lt.fp64_configs()
    for cfg, name in enumerate(names):
        # TMA configs need even N, K; cp.async configs take ragged shapes
        M, N, K = (200, 136, 98) if name.startswith("tma") else (131, 77, 45)
        A, B, C0 = oracle_mod.make_problem(M, N, K, phi=4, seed=cfg)
        C = run_fp64(cuda, A, B, C0, 1.5, 0.5, config=cfg)
        Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
        check(C, Cref, den, K, cublas_error(cuda, A, B, C0, 1.5, 0.5, Cref, den), name)


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (3, 5, 7), (129, 65, 33), (64, 200, 1000), (257, 3, 64)])
def test_ragged_shapes(cuda, oracle_mod, M, N, K):
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=2, seed=M + N + K)
    C = run_fp64(cuda, A, B, C0, -0.5, 2.0)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, -0.5, 2.0)
    check(C, Cref, den, K, cublas_error(cuda, A, B, C0, -0.5, 2.0, Cref, den))


@pytest.mark.parametrize("M,N,K,offset,beta", [(256, 256, 8192, 0, 0.5), (1024, 64, 4096, 0, 0.0),
                                               (300, 130, 5000, 1, 1.0), (128, 96, 2047, 0, -1.0)])
def test_k_split_shapes(cuda, oracle_mod, M, N, K, offset, beta):
    """Few tiles and long K: the launch cuts K into ranges whose partial sums are reduced in a
    second kernel (TMA and cp.async staging, ragged edges, odd K, beta = 0 not reading C)."""
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=3, seed=M + K)
    if beta == 0.0:
        C0 = np.full_like(C0, np.nan)
    C = run_fp64(cuda, A, B, C0, 1.25, beta, offset=offset)
    Cref, den = oracle_mod.dot2_rows(A, B, None if beta == 0.0 else C0, 1.25, beta)
    check(C, Cref, den, K, cublas_error(cuda, A, B, C0, 1.25, beta, Cref, den))


@pytest.mark.parametrize("M,N,K,offset,beta", [(64, 64, 8192, 0, 0.5), (130, 70, 3001, 1, -1.0),
                                               (700, 500, 2048, 0, 0.0)])
def test_stream_k_every_config(cuda, oracle_mod, M, N, K, offset, beta):
    """Stream-K: few tiles against 148 SMs, so the k-block iterations are dealt out in equal ranges
    and tiles shared by several CTAs (at 64x64x8192 one tile by all of them) are summed in K order by
    the fix-up kernel; every tile configuration the pointers allow, ragged edges and odd K."""
    import libthom_b200 as lt

    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=3, seed=3 * M + K)
    if beta == 0.0:
        C0 = np.full_like(C0, np.nan)
    Cref, den = oracle_mod.dot2_rows(A, B, None if beta == 0.0 else C0, 0.75, beta)
    e_cublas = cublas_error(cuda, A, B, C0, 0.75, beta, Cref, den)
    names = lt.fp64_configs()
    for cfg, name in enumerate(names):
        if offset and name.startswith("tma"):
            continue  # TMA needs 16-byte aligned operands and even pitches
        C = run_fp64(cuda, A, B, C0, 0.75, beta, config=cfg, offset=offset)
        check(C, Cref, den, K, e_cublas, name)


def test_long_k_stream_k_at_4096_cubed(cuda, oracle_mod):
    """4096^3 with the default configuration: 256 k-blocks per 128x64 tile, where the schedule model
    takes stream-K for its modelled 2 % gain over the 13.84-wave whole-tile grid. Every CTA's range
    then starts and ends inside tiles, so about 2 x 148 tile pieces go through the fix-up. Checked on
    sampled rows against the compensated oracle, and against cuBLAS on the same inputs."""
    import libthom_b200 as lt

    torch = cuda
    n = 4096
    A, B, C0 = oracle_mod.make_problem(n, n, n, phi=2, seed=4096)
    rows = np.array([0, 1, 127, 128, 1337, 2048, 4000, n - 1])
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5, rows=rows)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    dC, dR = to_dev(torch, C0), to_dev(torch, C0)
    lt.dgemm_fp64(dA, dB, dC, n, n, n, 1.5, 0.5)
    lt.dgemm_cublas(dA, dB, dR, n, n, n, 1.5, 0.5)
    torch.cuda.synchronize()
    lt.device_status()
    C, R = dC.cpu().numpy(), dR.cpu().numpy()
    e_cublas = oracle_mod.componentwise_error(R[rows], Cref, den)[0]
    check(C[rows], Cref, den, n, e_cublas, "4096^3")
    # every element, not only the sampled rows: within the two kernels' summed error bars of cuBLAS
    scale = 1.5 * (np.abs(A) @ np.abs(B)) + 0.5 * np.abs(C0)
    assert np.all(np.abs(C - R) <= 2 * fp64_bound(n) * scale)


def test_unaligned_pointers_take_general_path(cuda, oracle_mod):
    M, N, K = 96, 64, 80
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=4)
    C = run_fp64(cuda, A, B, C0, 1.0, 1.0, offset=1)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 1.0)
    check(C, Cref, den, K, cublas_error(cuda, A, B, C0, 1.0, 1.0, Cref, den))


def test_k_zero_and_beta_zero(cuda, oracle_mod):
    A, B, C0 = oracle_mod.make_problem(20, 30, 10, seed=1)
    C = run_fp64(cuda, np.zeros((20, 0)), np.zeros((0, 30)), C0, 2.0, 0.25)
    assert np.array_equal(C, 0.25 * C0)
    # beta == 0: C is not read, so NaN garbage in C does not leak into the result
    garbage = np.full((20, 30), np.nan)
    C = run_fp64(cuda, A, B, garbage, 1.0, 0.0)
    assert np.all(np.isfinite(C))


def test_config1_against_cublas(cuda, oracle_mod):
    """Plain 1024^3 DGEMM, alpha=1, beta=0, U[-1,1); checked against cuBLAS DGEMM (the
    reference's GPU oracle, routines/dgemm/dgemm_cublas_tc.cu) and the host oracles."""
    import libthom_b200 as lt

    torch = cuda
    n = 1024
    A, B, C0 = oracle_mod.make_problem(n, n, n, seed=1234)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    dC = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    dR = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    lt.dgemm_fp64(dA, dB, dC, n, n, n, 1.0, 0.0)
    lt.dgemm_cublas(dA, dB, dR, n, n, n, 1.0, 0.0)
    torch.cuda.synchronize()
    C, R = dC.cpu().numpy(), dR.cpu().numpy()
    rows = np.arange(0, n, 37)
    Cref, den = oracle_mod.dot2_rows(A, B, None, 1.0, 0.0, rows=rows)
    e_ours = oracle_mod.componentwise_error(C[rows], Cref, den)[0]
    e_cublas = oracle_mod.componentwise_error(R[rows], Cref, den)[0]
    assert e_ours <= fp64_bound(n) and e_cublas <= fp64_bound(n)
    assert e_ours <= tight_fp64_bound(e_cublas), (e_ours, e_cublas)
    # agreement with cuBLAS within the sum of both errors' statistical bars
    assert oracle_mod.componentwise_error(C[rows], R[rows], den)[0] <= e_ours + e_cublas + 16 * U
    # blocked host oracle agrees too
    Cb = oracle_mod.dgemm_blocked(A, B, C0, 1.0, 0.0)
    assert oracle_mod.componentwise_error(C[rows], Cb[rows], den)[0] <= 2 * fp64_bound(n)


def test_reference_contract_wrapper_times(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    A, B, C0 = oracle_mod.make_problem(256, 256, 256, seed=2)
    dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    ms = lt.dgemm("tc100", dA, dB, dC, 256, 256, 256, 1.0, 1.0)
    assert ms > 0.0
    ms2 = lt.dgemm("cublas_tc", dA, dB, dC, 256, 256, 256, 1.0, 1.0)
    assert ms2 > 0.0
