"""GPU test of the allocation-free Ozaki DGEMM (lt_dgemm_ozaki_noalloc).

That entry point exists for callers that cannot allocate device memory — a framework whose own pool
owns the GPU, a service that must not allocate on its request path, a process under a hard memory
cap. Its scratch is a fixed device array inside the library, shared by every call, so this test
checks that two calls in a row (different shapes, different data: the second must not see the
first call's leftovers) give exactly what the allocating entry point lt_dgemm_ozaki gives — the
Ozaki path is bit-reproducible, so the tolerance is zero — and that a problem too large for the
array is refused. The file is named to run last, after every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu


def run_both(torch, oracle_mod, M, N, K, s, seed, alpha, beta):
    import libthom_b200 as lt

    L = lt.lib()
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=6, seed=seed, smax=5)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    c_ref, c_new = to_dev(torch, C0), to_dev(torch, C0)
    lt.check(L.lt_dgemm_ozaki(dA.data_ptr(), dB.data_ptr(), c_ref.data_ptr(), M, N, K, alpha, beta, s, None))
    lt.check(L.lt_dgemm_ozaki_noalloc(dA.data_ptr(), dB.data_ptr(), c_new.data_ptr(), M, N, K, alpha, beta, s, None))
    torch.cuda.synchronize()
    return c_new.cpu().numpy(), c_ref.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(cuda, oracle_mod):
    # a larger problem first, then a smaller one with other data: stale scratch would show
    first, ref1 = run_both(cuda, oracle_mod, 700, 520, 900, 8, seed=11, alpha=1.5, beta=0.5)
    second, ref2 = run_both(cuda, oracle_mod, 130, 257, 333, 7, seed=12, alpha=-1.0, beta=0.0)
    assert np.array_equal(first, ref1)
    assert np.array_equal(second, ref2)
    assert np.all(np.isfinite(first)) and np.all(np.isfinite(second))


def test_noalloc_rejects_problems_beyond_the_static_scratch(cuda):
    import libthom_b200 as lt

    L = lt.lib()
    M = N = K = 4096  # needs about 8 * (32 + 32) * 128 * 4 KB = 268 MB with 8 slices
    assert L.lt_ozaki_workspace_size(M, N, K, 8) > (32 << 20)
    rc = L.lt_dgemm_ozaki_noalloc(0x1000, 0x1000, 0x1000, M, N, K, 1.0, 0.0, 8, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT
    assert b"static scratch" in L.lt_last_error_message()
