"""Failure detection on the GPU without a fault: a bounded device wait that runs out.

Every pipeline wait in the kernels is bounded (lt_common.cuh: mbar_wait); when a stage never
completes, the waiting warp records LT_ERR_DEVICE_TIMEOUT in the device error word, raises the
CTA's abort flag so the other roles leave their loops, and the kernel returns. The self-test waits
on a barrier that nothing arrives at, with a 50 ms limit, and checks that the host reads the
status and that the context keeps working.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import fp64_bound, to_dev

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_survives(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    assert L.lt_check_device_status() == lt.LT_OK
    lt.check(L.lt_selftest_wait_timeout(50.0, None))
    torch.cuda.synchronize()
    rc = L.lt_check_device_status()
    assert rc == lt.LT_ERR_DEVICE_TIMEOUT
    assert b"tag 99" in L.lt_last_error_message(), L.lt_last_error_message()
    assert L.lt_check_device_status() == lt.LT_OK  # reading the word clears it
    # the context is intact: a DGEMM right after runs and is correct
    A, B, C0 = oracle_mod.make_problem(96, 80, 64, seed=12)
    dA, dB, dC = to_dev(torch, A), to_dev(torch, B), to_dev(torch, C0)
    lt.dgemm_fp64(dA, dB, dC, 96, 80, 64, 1.0, 0.5)
    torch.cuda.synchronize()
    lt.device_status()
    Cref, den = oracle_mod.dot2_rows(A, B, C0, 1.0, 0.5)
    assert oracle_mod.componentwise_error(dC.cpu().numpy(), Cref, den)[0] <= fp64_bound(64)
