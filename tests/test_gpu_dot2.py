"""GPU parity of lt_dot2_rows, the library's compensated (double-double) reference of sampled rows
that bench.py uses to measure componentwise errors: bit-identical to the CPU oracle's Dot2
(oracle_dgemm_dot2_rows: error-free products, double-double sums in k order, one final rounding),
denominators included."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,phi,alpha,beta", [(100, 70, 300, 8, 1.5, 0.5), (33, 300, 1, 0, -1.0, 2.0),
                                                  (64, 129, 4096, 32, 1.0, 0.0), (5, 3, 777, 60, 0.75, -0.25)])
def test_dot2_rows_bit_exact(cuda, oracle_mod, M, N, K, phi, alpha, beta):
    import libthom_b200 as lt

    torch = cuda
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=phi, seed=M + K)
    rows = np.unique(np.linspace(0, M - 1, min(M, 17)).astype(np.int64))
    Cref, den = oracle_mod.dot2_rows(A, B, None if beta == 0.0 else C0, alpha, beta, rows=rows)
    dA, dB, dC0 = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    rows_d = torch.from_numpy(rows).cuda()
    gC = torch.empty(len(rows), N, dtype=torch.float64, device="cuda")
    gD = torch.empty_like(gC)
    lt.dot2_rows(dA, dB, dC0 if beta != 0.0 else None, M, N, K, alpha, beta, rows_d, gC, gD)
    torch.cuda.synchronize()
    lt.device_status()
    assert np.array_equal(gC.cpu().numpy(), Cref)
    assert np.array_equal(gD.cpu().numpy(), den)


def test_componentwise_error_against_device_reference(cuda, oracle_mod):
    """The on-device error measurement (lt_dot2_rows + lt_componentwise_error) gives the oracle's
    number for the native FP64 kernel's result."""
    import libthom_b200 as lt

    torch = cuda
    M, N, K = 96, 80, 500
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=4, seed=3)
    dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    dC0 = to_dev(torch, C0)
    lt.dgemm_fp64(dA, dB, dC, M, N, K, 1.5, 0.5)
    rows = np.arange(0, M, 5, dtype=np.int64)
    rows_d = torch.from_numpy(rows).cuda()
    gC = torch.empty(len(rows), N, dtype=torch.float64, device="cuda")
    gD = torch.empty_like(gC)
    lt.dot2_rows(dA, dB, dC0, M, N, K, 1.5, 0.5, rows_d, gC, gD)
    err_dev = lt.componentwise_error(dC[rows_d].contiguous(), gC, gD, gC.numel())[0]
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.5, 0.5, rows=rows)
    err_cpu = oracle_mod.componentwise_error(dC.cpu().numpy()[rows], Cref, den)[0]
    assert err_dev == err_cpu
