"""GPU checks of lt_dgemm_auto (the faster of native FP64 and Ozaki per call).

Whichever form the cost model picks, the result is bit-identical to calling that form directly
(lt_dgemm_fp64, or lt_dgemm_ozaki with the selector's slice count), and within the FP64
componentwise bound (K + 4) u of the compensated oracle on sampled rows.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import fp64_bound

pytestmark = pytest.mark.gpu


def make(torch, M, N, K, seed):
    import libthom_b200 as lt

    A = torch.empty(M, K, dtype=torch.float64, device="cuda")
    B = torch.empty(K, N, dtype=torch.float64, device="cuda")
    C0 = torch.empty(M, N, dtype=torch.float64, device="cuda")
    lt.fill(A, M * K, seed, 0)
    lt.fill(B, K * N, seed, 1)
    lt.fill(C0, M * N, seed, 2)
    return A, B, C0


@pytest.mark.parametrize("M,N,K,expect", [(2048, 2048, 2048, "ozaki"), (16384, 64, 1024, "fp64"),
                                          (300, 200, 100, "fp64"), (4096, 4096, 1024, "ozaki")])
def test_auto_matches_the_chosen_form(cuda, M, N, K, expect):
    import libthom_b200 as lt

    torch = cuda
    A, B, C0 = make(torch, M, N, K, seed=77)
    C = C0.clone()
    form, s = lt.dgemm_auto(A, B, C, M, N, K, 1.5, 0.5)
    torch.cuda.synchronize()
    lt.device_status()
    assert form == (lt.LT_FORM_OZAKI if expect == "ozaki" else lt.LT_FORM_FP64), (form, s)
    R = C0.clone()
    if form == lt.LT_FORM_OZAKI:
        assert 3 <= s <= 10
        lt.dgemm_ozaki(A, B, R, M, N, K, 1.5, 0.5, slices=s)
    else:
        assert s == 0
        lt.dgemm_fp64(A, B, R, M, N, K, 1.5, 0.5)
    torch.cuda.synchronize()
    assert torch.equal(C, R)
    rows = torch.tensor(np.linspace(0, M - 1, 8).astype(np.int64), device="cuda")
    Cref = torch.empty(8, N, dtype=torch.float64, device="cuda")
    den = torch.empty(8, N, dtype=torch.float64, device="cuda")
    lt.dot2_rows(A, B, C0, M, N, K, 1.5, 0.5, rows, Cref, den)
    err, _ = lt.componentwise_error(C[rows].contiguous(), Cref, den, 8 * N)
    assert err <= fp64_bound(K), err


def test_auto_registry_entry_and_empty_shapes(cuda):
    import libthom_b200 as lt

    torch = cuda
    M, N, K = 512, 256, 128
    A, B, C0 = make(torch, M, N, K, seed=5)
    C = C0.clone()
    ms = lt.dgemm("auto", A, B, C, M, N, K, 1.0, 0.0)
    assert ms > 0.0
    R = C0.clone()
    lt.dgemm_fp64(A, B, R, M, N, K, 1.0, 0.0)
    torch.cuda.synchronize()
    assert torch.equal(C, R)
    # K = 0: C = beta * C0
    C = C0.clone()
    form, s = lt.dgemm_auto(A, B, C, M, N, 0, 1.0, 0.5)
    torch.cuda.synchronize()
    assert form == lt.LT_FORM_FP64 and s == 0
    assert torch.equal(C, 0.5 * C0)
