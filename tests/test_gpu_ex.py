"""lt_dgemm_ex: row strides and transposed operands, both forms.

Every matrix is stored with a padded row stride whose padding holds NaN: no kernel may read it (a NaN
read would poison the result) and C's padding must come back untouched. Ozaki form: bit-identical to
the CPU restatement on the packed op(A), op(B) (a transposed operand goes through the other side's
split kernels, which write the same digits). FP64 form: within the (K + 4) u componentwise bound of
the compensated oracle (odd strides take the cp.async staging, even ones TMA, transposes a packing
pre-pass).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import fp64_bound

pytestmark = pytest.mark.gpu


def padded(X, pad):
    rows, cols = X.shape
    P = np.full((rows, cols + pad), np.nan)
    P[:, :cols] = X
    return P


@pytest.mark.parametrize("form", ["fp64", "ozaki"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("pad", [2, 3])
def test_strides_and_transposes(cuda, oracle_mod, form, ta, tb, pad):
    import libthom_b200 as lt

    torch = cuda
    M, N, K = 150, 130, 96
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=3, seed=M + 7 * pad + (ta == "T") + 2 * (tb == "T"))
    As = padded(A.T.copy() if ta == "T" else A, pad)
    Bs = padded(B.T.copy() if tb == "T" else B, pad)
    Cs = padded(C0, pad + 1)
    dA, dB, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (As, Bs, Cs))
    alpha, beta = 1.25, -0.5
    f = lt.LT_FORM_OZAKI if form == "ozaki" else lt.LT_FORM_FP64
    lt.dgemm_ex(ta, tb, M, N, K, alpha, dA, As.shape[1], dB, Bs.shape[1], beta, dC, Cs.shape[1], form=f, slices=7)
    torch.cuda.synchronize()
    lt.device_status()
    out = dC.cpu().numpy()
    assert np.all(np.isnan(out[:, N:])), "padding of C was written"
    C = out[:, :N]
    if form == "ozaki":
        R = oracle_mod.ozaki_dgemm(A, B, C0, alpha, beta, 7)
        assert np.array_equal(C, R), np.abs(C - R).max()
    else:
        Cref, den = oracle_mod.dot2_rows(A, B, C0, alpha, beta)
        assert oracle_mod.componentwise_error(C, Cref, den)[0] <= fp64_bound(K)


def test_long_k_split_with_strides(cuda, oracle_mod):
    """FP64 form, few tiles and long K (the K split and its reduction run with ldc != N)."""
    import libthom_b200 as lt

    torch = cuda
    M, N, K = 128, 96, 6000
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=2, seed=5)
    As, Bs, Cs = padded(A, 4), padded(B, 2), padded(C0, 6)
    dA, dB, dC = (torch.from_numpy(x).cuda() for x in (As, Bs, Cs))
    lt.dgemm_ex("N", "N", M, N, K, 1.0, dA, As.shape[1], dB, Bs.shape[1], 1.0, dC, Cs.shape[1])
    torch.cuda.synchronize()
    out = dC.cpu().numpy()
    assert np.all(np.isnan(out[:, N:]))
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 1.0)
    assert oracle_mod.componentwise_error(out[:, :N], Cref, den)[0] <= fp64_bound(K)
