"""GPU accuracy at the benchmark configurations' own shapes (sampled rows, compensated reference on the
device, lt_dot2_rows, itself bit-identical to the CPU oracle's Dot2):

- 65536 x 64 x 4096 and 2048 x 2048 x 65536 with rows of A and columns of B scaled by 2^s,
  s ~ U{-64..64} (the tall and long-K configuration);
- 2048^3 with entries u 2^e, e ~ U{-32..32} (the widest exponent spread of the square configuration).

Native FP64: within the worst-case bound and the statistical bar (four times cuBLAS's error on the same
rows). CRT form: with the modulus count the benchmark picks for these data, no worse than native FP64.
Slice form: with s = 7 (s = 8 at phi = 32), no worse than native FP64.
"""
from __future__ import annotations

import pytest

from conftest import fp64_bound, tight_fp64_bound

pytestmark = pytest.mark.gpu

SEED = 1234


def setup(torch, lt, M, N, K, phi, smax, alpha, beta, nrows=8):
    dev = torch.device("cuda")
    A = torch.empty(M, K, dtype=torch.float64, device=dev)
    B = torch.empty(K, N, dtype=torch.float64, device=dev)
    C0 = torch.empty(M, N, dtype=torch.float64, device=dev)
    lt.fill(A, M * K, SEED, 1, phi)
    lt.fill(B, K * N, SEED, 2, phi)
    lt.fill(C0, M * N, SEED, 3, phi)
    if smax:
        lt.scale_rows(A, M, K, SEED, 4, smax)
        lt.scale_cols(B, K, N, SEED, 5, smax)
    rows = torch.linspace(0, M - 1, nrows, device=dev).round().to(torch.int64)
    Cref = torch.empty(nrows, N, dtype=torch.float64, device=dev)
    den = torch.empty_like(Cref)
    lt.dot2_rows(A, B, C0, M, N, K, alpha, beta, rows, Cref, den)
    torch.cuda.synchronize()

    def err(fn):
        C = C0.clone()
        fn(C)
        torch.cuda.synchronize()
        lt.device_status()
        return lt.componentwise_error(C[rows].contiguous(), Cref, den, Cref.numel())[0]

    return A, B, err


@pytest.mark.parametrize("M,N,K,phi,smax,alpha,beta,moduli,slices", [
    (65536, 64, 4096, 0, 64, 1.0, 0.0, 15, 7),
    (2048, 2048, 65536, 0, 64, 1.0, 0.0, 15, 7),
    (2048, 2048, 2048, 32, 0, 1.5, 0.5, 16, 8),
])
def test_configuration_accuracy(cuda, M, N, K, phi, smax, alpha, beta, moduli, slices):
    import libthom_b200 as lt

    torch = cuda
    A, B, err = setup(torch, lt, M, N, K, phi, smax, alpha, beta)
    e64 = err(lambda C: lt.dgemm_fp64(A, B, C, M, N, K, alpha, beta))
    ecb = err(lambda C: lt.dgemm_cublas(A, B, C, M, N, K, alpha, beta))
    assert e64 <= fp64_bound(K) and ecb <= fp64_bound(K)
    assert e64 <= tight_fp64_bound(ecb), (e64, ecb)
    ecrt = err(lambda C: lt.dgemm_ozaki_crt(A, B, C, M, N, K, alpha, beta, moduli))
    assert ecrt <= e64, (ecrt, e64)
    esl = err(lambda C: lt.dgemm_ozaki(A, B, C, M, N, K, alpha, beta, slices))
    assert esl <= e64, (esl, e64)
