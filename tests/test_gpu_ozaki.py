"""GPU parity of the Ozaki INT8-slice DGEMM (lt_dgemm_ozaki / dgemm_ozaki<s>).

Oracle: oracle_ozaki_dgemm, a CPU restatement with the same arithmetic in the same order, so the
GPU result must be bit-identical (integer slice products are exact; every FP64 step is
specified). Accuracy against the compensated Dot2 oracle is checked separately.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import U, fp64_bound, to_dev

pytestmark = pytest.mark.gpu


def run_ozaki(torch, A, B, C0, alpha, beta, s, workspace=None):
    import libthom_b200 as lt

    M, K = A.shape
    N = B.shape[1]
    dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    lt.dgemm_ozaki(dA, dB, dC, M, N, K, alpha, beta, slices=s, workspace=workspace)
    torch.cuda.synchronize()
    lt.device_status()
    return dC.cpu().numpy().reshape(M, N)


def assert_bit_exact(C, R):
    same = (C == R) | (np.isnan(C) & np.isnan(R))
    if not same.all():
        idx = np.argwhere(~same)[:5]
        raise AssertionError(f"{(~same).sum()} mismatches, first {[(tuple(i), C[tuple(i)], R[tuple(i)]) for i in idx]}")


@pytest.mark.parametrize("s", [1, 3, 5, 8, 10, 12])
def test_bit_exact_vs_restatement(cuda, oracle_mod, s):
    M, N, K = 200, 150, 300
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=8, seed=s)
    C = run_ozaki(cuda, A, B, C0, 1.5, 0.5, s)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, 1.5, 0.5, s))


def _digit_edge_matrix(rng, rows, cols, by_rows):
    """Entries that drive the balanced base-256 digits to their edges: each row (or column) holds
    its maximum just below a power of two (top digit +-64) or exactly at one (frexp puts it at
    0.5 2^e), values whose lower digits are all -128 or all 127 (V = +-(2^(8s-2) - 1)-like bit
    patterns: 1 - 2^-k), tiny values and subnormals far below the maximum, exact zeros, and both
    signs."""
    X = rng.uniform(-1.0, 1.0, size=(rows, cols))
    lines = X if by_rows else X.T
    specials = np.array([1.0 - 2.0 ** -53, -(1.0 - 2.0 ** -53), 0.5, -0.5, 1.0 - 2.0 ** -20, -(1.0 - 2.0 ** -30),
                         2.0 ** -60, -(2.0 ** -60), 5e-324, -5e-324, 2.2250738585072014e-308, 0.0,
                         0.75 + 2.0 ** -40, -(0.5 + 2.0 ** -52), 2.0 ** -8 - 2.0 ** -61, -(2.0 ** -16)])
    for i in range(lines.shape[0]):
        idx = rng.choice(lines.shape[1], size=min(len(specials), lines.shape[1]), replace=False)
        lines[i, idx] = specials[: len(idx)] * (2.0 ** int(rng.integers(-40, 41)))
        if i % 3 == 0:
            lines[i] *= 2.0 ** int(rng.integers(-900, 900))  # whole line far from 1
    return X


@pytest.mark.parametrize("s", [1, 2, 7, 8, 9, 12])
def test_digit_edges_bit_exact(cuda, oracle_mod, s):
    """Digit extraction at its boundaries, on both integer widths of the GPU split (64-bit up to
    s = 8, 128-bit above), for the row (A) and column (B) split kernels alike."""
    rng = np.random.default_rng(100 + s)
    M, N, K = 150, 140, 96
    A = _digit_edge_matrix(rng, M, K, by_rows=True)
    B = _digit_edge_matrix(rng, K, N, by_rows=False)
    C0 = rng.uniform(-1.0, 1.0, size=(M, N))
    C = run_ozaki(cuda, A, B, C0, 1.25, -0.5, s)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, 1.25, -0.5, s))


@pytest.mark.parametrize("M,N,K", [(1, 1, 1), (129, 130, 33), (127, 255, 64), (64, 17, 1000), (300, 8, 96)])
def test_ragged_shapes_bit_exact(cuda, oracle_mod, M, N, K):
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=3, seed=M * 7 + N)
    C = run_ozaki(cuda, A, B, C0, -1.0, 0.75, 7)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, -1.0, 0.75, 7))


@pytest.mark.parametrize("M,N,K,s", [(256, 128, 64, 8), (300, 200, 96, 7), (129, 64, 40, 5), (1536, 1664, 32, 3),
                                     (260, 24, 17000, 8)])
def test_cta_pair_kernel_bit_exact(cuda, oracle_mod, M, N, K, s):
    """Problems with two or more 128-row blocks run on the CTA-pair kernel (tcgen05 cta_group::2,
    256 x 128 tiles): an odd row-block count (the last pair's second CTA holds no rows of A), more
    tiles than CTA pairs (persistent loop), and K long enough for two INT32-safe groups."""
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=5, seed=M + 3 * N + s)
    C = run_ozaki(cuda, A, B, C0, 1.25, -0.5, s)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, 1.25, -0.5, s))


@pytest.mark.parametrize("M,N,K,beta,pinned", [(1000, 300, 200, 0.5, True), (300, 130, 96, 0.0, False),
                                              (2560, 384, 64, 1.0, True), (2100, 200, 72, 0.5, True)])
def test_host_resident_bit_exact(cuda, oracle_mod, M, N, K, beta, pinned):
    """lt_dgemm_ozaki_host: operands in host memory, streamed through the GPU in row panels (a
    ragged last panel, pageable and pinned buffers, beta = 0 skipping the C0 copy): the same bits
    as the oracle, and C0 is only read when beta != 0."""
    import libthom_b200 as lt

    torch = cuda
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=4, seed=M + N + K)
    Ah, Bh = torch.from_numpy(A.copy()), torch.from_numpy(B.copy())
    Ch = torch.from_numpy(C0.copy() if beta != 0.0 else np.full((M, N), np.nan))
    if pinned:
        Ah, Bh, Ch = Ah.pin_memory(), Bh.pin_memory(), Ch.pin_memory()
    lt.dgemm_ozaki_host(Ah, Bh, Ch, M, N, K, 1.5, beta, slices=6)
    lt.device_status()
    assert_bit_exact(Ch.numpy(), oracle_mod.ozaki_dgemm(A, B, C0, 1.5, beta, 6))


def test_long_k_multiple_groups(cuda, oracle_mod):
    """K = 20000 > 16640 (the INT32-safe group length of an 8-pair diagonal): two groups."""
    M, N, K = 64, 48, 20000
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=77, smax=8)
    C = run_ozaki(cuda, A, B, C0, 1.0, 0.0, 8)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 0.0, 8))


def test_nan_inf_zero(cuda, oracle_mod):
    M, N, K = 40, 30, 64
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=9)
    A[3, 7] = np.nan
    B[11, 5] = np.inf
    A[6, :] = 0.0
    B[:, 9] = 0.0
    C = run_ozaki(cuda, A, B, C0, 1.0, 0.5, 6)
    R = oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 0.5, 6)
    assert_bit_exact(C, R)
    assert np.all(np.isnan(C[3, :])) and np.all(np.isnan(C[:, 5]))


def test_accuracy_reaches_fp64(cuda, oracle_mod):
    """Eight slices on unscaled data: componentwise error within the FP64 bound."""
    M, N, K = 256, 256, 1024
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=1234)
    C = run_ozaki(cuda, A, B, C0, 1.5, 0.5, 8)
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5)
    err = oracle_mod.componentwise_error(C, Cref, den)
    assert err[0] <= fp64_bound(K), err


def test_caller_workspace(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    M, N, K, s = 96, 80, 200, 5
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=31)
    need = lt.ozaki_workspace_size(M, N, K, s)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    C = run_ozaki(torch, A, B, C0, 1.0, 1.0, s, workspace=ws)
    assert_bit_exact(C, oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 1.0, s))
    small = torch.empty(need - 256, dtype=torch.uint8, device="cuda")
    with pytest.raises(lt.LtError) as ei:
        run_ozaki(torch, A, B, C0, 1.0, 1.0, s, workspace=small)
    assert ei.value.code == lt.LT_ERR_NO_MEMORY


def test_reference_contract_wrappers(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    M = N = K = 128
    A, B, C0 = oracle_mod.make_problem(M, N, K, seed=3)
    for s in range(3, 11):
        dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
        ms = lt.dgemm(f"ozaki{s}", dA, dB, dC, M, N, K, 1.0, 1.0)
        assert ms > 0
        assert_bit_exact(dC.cpu().numpy(), oracle_mod.ozaki_dgemm(A, B, C0, 1.0, 1.0, s))
