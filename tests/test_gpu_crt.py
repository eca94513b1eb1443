"""GPU parity of the CRT form (Ozaki scheme II): bit-identical to the CPU restatement
(oracle_crt_dgemm) on ragged shapes, every limb count, alpha/beta, exponent spread, row/column
scaling, non-finite and zero rows, K = 0 and a K long enough to need two INT32 accumulation groups;
rows and columns at the edges of the norm-bound scaling; the entry points agree with each other; and
at 2048^3 the error against the compensated reference is no worse than the native FP64 kernel's on the
same sampled rows."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu

CASES = [
    # M, N, K, phi, smax, alpha, beta, moduli
    (300, 260, 500, 0, 0, 1.5, 0.5, 15),
    (256, 256, 256, 8, 0, 1.0, 0.0, 14),
    (129, 513, 1000, 32, 0, -0.5, 2.0, 16),
    (64, 40, 3000, 0, 64, 1.0, 1.0, 17),
    (520, 130, 129, 4, 0, 1.0, -1.0, 20),
    (700, 300, 64, 0, 0, 2.0, 0.0, 8),
    (333, 77, 200, 2, 0, 1.0, 0.5, 10),
    (1, 1, 1, 0, 0, 1.0, 0.5, 15),
    (1, 300, 7, 3, 0, 1.0, 0.0, 15),
    (600, 1, 33, 0, 5, 1.0, 0.25, 18),
    (257, 255, 4096, 0, 0, 1.0, 0.0, 15),
]


def run_crt(torch, A, B, C0, alpha, beta, n):
    import libthom_b200 as lt

    M, K = A.shape
    N = B.shape[1]
    dC = to_dev(torch, C0)
    lt.dgemm_ozaki_crt(to_dev(torch, A), to_dev(torch, B), dC, M, N, K, alpha, beta, n)
    torch.cuda.synchronize()
    lt.device_status()
    return dC.cpu().numpy()


@pytest.mark.parametrize("M,N,K,phi,smax,alpha,beta,n", CASES)
def test_crt_bit_identical_to_restatement(cuda, oracle_mod, M, N, K, phi, smax, alpha, beta, n):
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=M + N + K, smax=smax)
    got = run_crt(cuda, A, B, C0, alpha, beta, n)
    want = oracle_mod.crt_dgemm(A, B, C0, alpha, beta, n)
    assert np.array_equal(got, want), f"max diff {np.max(np.abs(got - want))}"


def test_crt_nonfinite_zero_rows_and_k_zero(cuda, oracle_mod):
    A, B, C0 = oracle_mod.make_problem(300, 270, 90, seed=5)
    A[7, 11] = np.nan
    A[8, :] = 0.0
    A[9, 2] = -np.inf
    B[3, 200] = np.inf
    got = run_crt(cuda, A, B, C0, 1.25, -0.75, 15)
    want = oracle_mod.crt_dgemm(A, B, C0, 1.25, -0.75, 15)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.array_equal(got[~np.isnan(want)], want[~np.isnan(want)])
    assert np.all(np.isnan(got[7])) and np.all(np.isnan(got[:, 200]))
    # K = 0: C = beta C0 (alpha * 0 when beta = 0)
    import libthom_b200 as lt

    torch = cuda
    dC = to_dev(torch, C0)
    z = torch.zeros(8, dtype=torch.float64, device="cuda")
    lt.dgemm_ozaki_crt(z, z, dC, 300, 270, 0, 2.0, 0.5, 15)
    torch.cuda.synchronize()
    assert np.array_equal(dC.cpu().numpy(), 0.5 * C0)


@pytest.mark.parametrize("K", [1, 511, 512, 1100])
def test_crt_scaling_edges(cuda, oracle_mod, K):
    """Rows of A and columns of B that stress the integer norm bounds: subnormal-only, near the top of
    the double range, tiny normal, chunks of 512 at very different scales, a single nonzero entry in
    the last (partial) chunk, all zero; bit-identical to the restatement."""
    rng = np.random.default_rng(K)
    M, N = 40, 36
    A = rng.uniform(-1, 1, (M, K))
    B = rng.uniform(-1, 1, (K, N))
    C0 = rng.uniform(-1, 1, (M, N))
    A[0] *= 2.0 ** -1070
    A[1] *= 2.0 ** 1000
    A[2] *= 2.0 ** -1000
    A[3, : K // 2] *= 2.0 ** -700
    A[4] = 0.0
    A[4, K - 1] = -0.5
    A[5] = 0.0
    A[6] *= np.exp2(rng.integers(-300, 301, K))
    B[:, 0] *= 2.0 ** -1070
    B[:, 1] *= 2.0 ** -20
    B[: K // 2, 2] *= 2.0 ** 600
    B[:, 3] = 0.0
    B[K - 1, 3] = 3.0
    B[:, 4] *= np.exp2(rng.integers(-300, 301, K))
    for n in (14, 15, 17):
        got = run_crt(cuda, A, B, C0, 1.0, 0.5, n)
        want = oracle_mod.crt_dgemm(A, B, C0, 1.0, 0.5, n)
        assert np.array_equal(got, want, equal_nan=True), (n, np.nanmax(np.abs(got - want)))


@pytest.mark.slow
def test_crt_two_accumulation_groups(cuda, oracle_mod):
    """K above 1023 * 128 = 130944: each modulus accumulates in two INT32 groups whose residues the
    drain combines; still bit-identical."""
    M, N, K = 40, 300, 131200
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=77)
    got = run_crt(cuda, A, B, C0, 1.0, 0.5, 15)
    want = oracle_mod.crt_dgemm(A, B, C0, 1.0, 0.5, 15)
    assert np.array_equal(got, want)


def test_crt_entry_points_agree(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    M, N, K, n = 384, 320, 700, 15
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=2, seed=8)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    ref = run_crt(torch, A, B, C0, 1.5, 0.5, n)
    ws = torch.empty(lt.ozaki_crt_workspace_size(M, N, K, n), dtype=torch.uint8, device="cuda")
    c1 = to_dev(torch, C0)
    lt.dgemm_ozaki_crt(dA, dB, c1, M, N, K, 1.5, 0.5, n, workspace=ws)
    c2 = to_dev(torch, C0)
    lt.ozaki_crt_split(dA, dB, M, N, K, n, ws)
    lt.ozaki_crt_product(c2, M, N, K, 1.5, 0.5, n, ws)
    c3 = to_dev(torch, C0)
    ms = lt.dgemm("ozaki_crt15", dA, dB, c3, M, N, K, 1.5, 0.5)
    c4 = to_dev(torch, C0)
    lt.ozaki_crt_split(dA, dB, M, N, K, n, ws)
    lt.ozaki_crt_multiply(M, N, K, n, ws)
    lt.ozaki_crt_reconstruct(c4, M, N, K, 1.5, 0.5, n, ws)
    torch.cuda.synchronize()
    lt.device_status()
    assert ms > 0.0
    for c in (c1, c2, c3, c4):
        assert np.array_equal(c.cpu().numpy(), ref)


def test_crt_accuracy_at_2048_against_native_fp64(cuda):
    """2048^3, alpha = 1.5, beta = 0.5, U[-1,1) entries: with 14 moduli the max componentwise error on
    sampled rows (compensated reference computed on the device) is no worse than the native FP64
    kernel's on the same rows."""
    import libthom_b200 as lt

    torch = cuda
    n = 2048
    A = torch.empty(n, n, dtype=torch.float64, device="cuda")
    B, C0 = torch.empty_like(A), torch.empty_like(A)
    lt.fill(A, n * n, 1234, 1, 0)
    lt.fill(B, n * n, 1234, 2, 0)
    lt.fill(C0, n * n, 1234, 3, 0)
    rows = torch.arange(0, n, n // 8, dtype=torch.int64, device="cuda")
    Cref = torch.empty(rows.numel(), n, dtype=torch.float64, device="cuda")
    den = torch.empty_like(Cref)
    lt.dot2_rows(A, B, C0, n, n, n, 1.5, 0.5, rows, Cref, den)
    C = C0.clone()
    lt.dgemm_fp64(A, B, C, n, n, n, 1.5, 0.5)
    e64 = lt.componentwise_error(C[rows].contiguous(), Cref, den, Cref.numel())[0]
    C = C0.clone()
    lt.dgemm_ozaki_crt(A, B, C, n, n, n, 1.5, 0.5, 14)
    ecrt = lt.componentwise_error(C[rows].contiguous(), Cref, den, Cref.numel())[0]
    torch.cuda.synchronize()
    lt.device_status()
    assert ecrt <= e64, (ecrt, e64)


def test_crt_host_resident_path(cuda, oracle_mod):
    """lt_dgemm_ozaki_crt_host on pinned host buffers (row panels of A pipelined through the GPU) is
    bit-identical to the device-resident call, with several panels, ragged edges and K = 0."""
    import libthom_b200 as lt

    torch = cuda
    for (M, N, K) in [(1100, 300, 257), (70, 90, 0)]:
        A, B, C0 = oracle_mod.make_problem(M, N, max(K, 1), phi=3, seed=M)
        A, B = A[:, :K].copy(), B[:K, :].copy()
        ref = run_crt(torch, A, B, C0, 1.5, 0.5, 15) if K > 0 else 0.5 * C0
        Ah = torch.from_numpy(A).pin_memory()
        Bh = torch.from_numpy(B).pin_memory()
        Ch = torch.from_numpy(C0.copy()).pin_memory()
        lt.dgemm_ozaki_crt_host(Ah.data_ptr(), Bh.data_ptr(), Ch.data_ptr(), M, N, K, 1.5, 0.5, 15)
        lt.device_status()
        assert np.array_equal(Ch.numpy(), ref)
