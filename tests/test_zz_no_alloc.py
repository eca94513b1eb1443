"""GPU test of the allocation-free Ozaki DGEMM (lt_dgemm_ozaki_noalloc).

That entry point exists for callers that cannot allocate device memory — a framework whose own pool
owns the GPU, a service that must not allocate on its request path, a process under a hard memory
cap. Its scratch is a fixed device array inside the library, shared by every call, so this test
checks that two calls in a row (different shapes, different data: the second must not see the
first call's leftovers) give exactly what the allocating entry point lt_dgemm_ozaki gives — the
Ozaki path is bit-reproducible, so the tolerance is zero — that a problem whose scratch just fits
the array runs and one just past it is refused, that K = 0 leaves beta*C0, and that a bounded
device wait giving up inside that path is reported by lt_check_device_status. The file is named to
run last, after every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu

NOALLOC_BYTES = 32 << 20  # LT_OZAKI_NOALLOC_BYTES


def run_both(torch, oracle_mod, M, N, K, s, seed, alpha, beta):
    import libthom_b200 as lt

    L = lt.lib()
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=6, seed=seed, smax=5)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    c_ref, c_new = to_dev(torch, C0), to_dev(torch, C0)
    lt.check(L.lt_dgemm_ozaki(dA.data_ptr(), dB.data_ptr(), c_ref.data_ptr(), M, N, K, alpha, beta, s, None))
    lt.check(L.lt_dgemm_ozaki_noalloc(dA.data_ptr(), dB.data_ptr(), c_new.data_ptr(), M, N, K, alpha, beta, s, None))
    torch.cuda.synchronize()
    lt.device_status()
    return c_new.cpu().numpy(), c_ref.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(cuda, oracle_mod):
    # a larger problem first, then a smaller one with other data: stale scratch would show
    first, ref1 = run_both(cuda, oracle_mod, 700, 520, 900, 8, seed=11, alpha=1.5, beta=0.5)
    second, ref2 = run_both(cuda, oracle_mod, 130, 257, 333, 7, seed=12, alpha=-1.0, beta=0.0)
    assert np.array_equal(first, ref1)
    assert np.array_equal(second, ref2)
    assert np.all(np.isfinite(first)) and np.all(np.isfinite(second))


def _largest_k_that_fits(L, M, N, s):
    """Largest K (multiple of 32) whose scratch fits the static array, found by the library's own
    size function, so the end of the array is the part this case reaches."""
    K = 32
    while L.lt_ozaki_workspace_size(M, N, K + 32, s) <= NOALLOC_BYTES:
        K += 32
    return K


def test_noalloc_at_the_size_limit(cuda, oracle_mod):
    import libthom_b200 as lt

    L = lt.lib()
    M, N, s = 637, 250, 7  # ragged edges, several 128-row blocks (the CTA-pair kernel)
    K = _largest_k_that_fits(L, M, N, s)
    assert NOALLOC_BYTES - L.lt_ozaki_workspace_size(M, N, K, s) < 64 << 10  # within 64 KB of the end
    got, ref = run_both(cuda, oracle_mod, M, N, K, s, seed=21, alpha=0.75, beta=-1.25)
    assert np.array_equal(got, ref)
    # one 32-deep chunk more does not fit: refused before any device work
    assert L.lt_ozaki_workspace_size(M, N, K + 32, s) > NOALLOC_BYTES
    rc = L.lt_dgemm_ozaki_noalloc(0x1000, 0x1000, 0x1000, M, N, K + 32, 1.0, 0.0, s, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT
    assert b"static scratch" in L.lt_last_error_message()


def test_noalloc_k_zero_leaves_beta_c0(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    M, N = 200, 130
    _, _, C0 = oracle_mod.make_problem(M, N, 8, seed=31)
    a = torch.zeros(8, dtype=torch.float64, device="cuda")  # any valid pointers: K = 0 reads no A or B
    dC = to_dev(torch, C0)
    lt.check(L.lt_dgemm_ozaki_noalloc(a.data_ptr(), a.data_ptr(), dC.data_ptr(), M, N, 0, 2.0, 0.5, 7, None))
    torch.cuda.synchronize()
    lt.device_status()
    assert np.array_equal(dC.cpu().numpy(), 0.5 * C0)


def test_noalloc_rejects_problems_beyond_the_static_scratch(cuda):
    import libthom_b200 as lt

    L = lt.lib()
    M = N = K = 4096  # needs about 8 * (32 + 32) * 128 * 4 KB = 268 MB with 8 slices
    assert L.lt_ozaki_workspace_size(M, N, K, 8) > NOALLOC_BYTES
    rc = L.lt_dgemm_ozaki_noalloc(0x1000, 0x1000, 0x1000, M, N, K, 1.0, 0.0, 8, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT
    assert b"static scratch" in L.lt_last_error_message()


def test_noalloc_reports_a_wait_that_gave_up(cuda, oracle_mod):
    """The allocation-free path's kernels report into a static error word of their own; a bounded
    wait that gives up there (the self-test: a barrier nothing arrives at, 50 ms limit) must reach
    the host through lt_check_device_status, and the path must keep working afterwards."""
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    assert L.lt_check_device_status() == lt.LT_OK
    lt.check(L.lt_selftest_wait_timeout_noalloc(50.0, None))
    torch.cuda.synchronize()
    assert L.lt_check_device_status() == lt.LT_ERR_DEVICE_TIMEOUT
    msg = L.lt_last_error_message()
    assert b"tag 99" in msg and b"allocation-free" in msg, msg
    assert L.lt_check_device_status() == lt.LT_OK  # reading the word clears it
    got, ref = run_both(cuda, oracle_mod, 300, 260, 500, 7, seed=41, alpha=1.0, beta=1.0)
    assert np.array_equal(got, ref)
