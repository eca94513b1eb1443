"""The reference's own HGEMM CUDA kernels, hgemm_final and hgemm_better_reuse
(routines/hgemm/hgemm_final.cu, routines/hgemm/hgemm_better_reuse.cu: mma.sync m16n8k16 with FP16
accumulation), compiled for sm_100a in oracle/_ref and run beside this library's tcgen05 kernel on
the same device buffers. They must pass the reference's own acceptance test against the oracle,
and this library's kernel must beat both at 8192^3 (the largest size of the reference's bench
list). The measured rates are printed (pytest -s); the reference kernels are never part of the
library."""
from __future__ import annotations

import numpy as np
import pytest

from test_gpu_hgemm import _reference_compare, dev

pytestmark = pytest.mark.gpu

ONE, ZERO = 0x3C00, 0x0000  # FP16 bit patterns of 1.0 and 0.0


@pytest.fixture(scope="module")
def ref_kernels():
    import oracle

    R = oracle.ref_hgemm_kernels_lib()
    if R is None:
        pytest.skip("reference HGEMM kernels not built (reference sources absent at build time)")
    return R


@pytest.mark.parametrize("name", ["ref_hgemm_final", "ref_hgemm_better_reuse"])
def test_reference_kernels_pass_their_acceptance_test(cuda, oracle_mod, ref_kernels, name):
    torch = cuda
    n = 1024  # a tile multiple for both kernels
    A, B, C0 = oracle_mod.make_half_problem(n, n, n, seed=1234)
    dA, dB, dC = dev(torch, A), dev(torch, B), dev(torch, C0)
    ms = getattr(ref_kernels, name)(dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), n, n, n, ONE, ZERO)
    torch.cuda.synchronize()
    assert ms > 0
    rows = np.arange(0, n, 61)
    C = dC.view(torch.int16).cpu().numpy().view(np.uint16).reshape(n, n)
    assert _reference_compare(C[rows], oracle_mod.hgemm_ref(A, B, C0, 1.0, 0.0, rows=rows)) == 0


def test_tc100_beats_reference_kernels_at_8192(cuda, oracle_mod, ref_kernels):
    import libthom_b200 as lt

    torch = cuda
    n = 8192
    g = torch.Generator(device="cuda").manual_seed(1234)
    A = torch.rand(n, n, device="cuda", generator=g).half()
    B = torch.rand(n, n, device="cuda", generator=g).half()
    C = torch.zeros(n, n, dtype=torch.float16, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    args = (A.data_ptr(), B.data_ptr(), C.data_ptr(), n, n, n, ONE, ZERO)
    t = {
        "reference hgemm_final": timed(lambda: ref_kernels.ref_hgemm_final(*args)),
        "reference hgemm_better_reuse": timed(lambda: ref_kernels.ref_hgemm_better_reuse(*args)),
        "cublas (FP16 accumulation)": timed(lambda: lt.hgemm_cublas(A, B, C, n, n, n, 1.0, 0.0, compute_f32=False)),
        "cublas (FP32 accumulation)": timed(lambda: lt.hgemm_cublas(A, B, C, n, n, n, 1.0, 0.0, compute_f32=True)),
        "tc100": timed(lambda: lt.hgemm_tc(A, B, C, n, n, n, 1.0, 0.0)),
    }
    lt.device_status()
    tf = {k: round(2.0 * n ** 3 / (v * 1e-3) / 1e12, 1) for k, v in t.items()}
    print("8192^3 HGEMM TFLOP/s:", tf)
    assert t["tc100"] < t["reference hgemm_final"] and t["tc100"] < t["reference hgemm_better_reuse"], tf
