"""GPU parity of the tcgen05 FP16 GEMM (hgemm_tc100 / lt_hgemm) of libthom's `hgemm` routine.

Oracle: the reference's own host check (routines/hgemm/hgemm.cu:135-149), restated in oracle/ and
pinned bit-exactly to the reference's compiled loop through tests/golden/hgemm_ref.npz, plus a
float64 evaluation of the same rows. Tolerance (floating point, FP32 accumulation in any order):
|C - exact| <= (2K + 4) 2^-24 den + 2^-11 |exact| + 2^-25, with den = |alpha| sum|a||b| + |beta||c|:
K FP32 additions whose rounding or truncation costs at most one FP32 ulp each, the epilogue's two
products and one sum, and the final rounding to FP16 (half an FP16 ulp; 2^-25 in the subnormal
range). Results whose exact value overflows FP16 must be Inf of the same sign.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

FP16_MAX_ROUND = 65520.0  # values at or above this round to Inf


def dev(torch, bits: np.ndarray, offset: int = 0):
    """FP16 device tensor holding the uint16 patterns `bits`, starting `offset` elements into its
    buffer (offset 1 leaves the data only 2-byte aligned)."""
    flat = torch.from_numpy(np.ascontiguousarray(bits).view(np.int16).ravel()).cuda()
    buf = torch.zeros(flat.numel() + offset, dtype=torch.int16, device="cuda")
    buf[offset:] = flat
    return buf[offset:].view(torch.float16)


def run_tc(torch, A, B, C0, alpha, beta, config=-1, offset=0):
    import libthom_b200 as lt

    M, K = A.shape
    N = B.shape[1]
    dA, dB, dC = dev(torch, A, offset), dev(torch, B, offset), dev(torch, C0, offset)
    lt.hgemm_tc(dA, dB, dC, M, N, K, alpha, beta, config=config)
    torch.cuda.synchronize()
    lt.device_status()
    return dC.view(torch.int16).cpu().numpy().view(np.uint16).reshape(M, N)


def tolerance(K, exact, den):
    return (2 * K + 4) * 2.0 ** -24 * den + 2.0 ** -11 * np.abs(exact) + 2.0 ** -25


def check_against_exact(oracle_mod, C, A, B, C0, alpha, beta, rows=None):
    """C (all rows, uint16) against the float64 value of the selected rows; returns the worst
    error relative to the tolerance."""
    K = A.shape[1]
    ex, den = oracle_mod.hgemm_exact_rows(A, B, C0, alpha, beta, rows=rows)
    got = (C if rows is None else C[rows]).view(np.float16).astype(np.float64)
    tol = tolerance(K, ex, den)
    over = np.abs(ex) >= FP16_MAX_ROUND + tol  # surely Inf
    under = np.abs(ex) < FP16_MAX_ROUND - tol  # surely finite
    assert np.array_equal(np.isinf(got) & over, over), "missing overflow to Inf"
    assert np.all(np.sign(got[over]) == np.sign(ex[over]))
    fin = under
    assert np.all(np.isfinite(got[fin])), "Inf/NaN where the result is finite"
    err = np.abs(got[fin] - ex[fin]) / tol[fin]
    return float(err.max()) if err.size else 0.0


def test_golden_cases(cuda, oracle_mod):
    g = np.load(ROOT / "tests" / "golden" / "hgemm_ref.npz")
    for i in range(int(g["ncases"][0])):
        alpha, beta = (float(x) for x in g[f"case{i}_scalars"])
        A, B, C0, Cref = g[f"case{i}_A"], g[f"case{i}_B"], g[f"case{i}_C0"], g[f"case{i}_C"]
        C = run_tc(cuda, A, B, C0, alpha, beta)
        assert check_against_exact(oracle_mod, C, A, B, C0, alpha, beta) <= 1.0, i
        # the reference loop's own output obeys the same bound: both within twice of each other
        K = A.shape[1]
        ex, den = oracle_mod.hgemm_exact_rows(A, B, C0, alpha, beta)
        a, r = C.view(np.float16).astype(np.float64), Cref.view(np.float16).astype(np.float64)
        both = np.isfinite(a) & np.isfinite(r)
        assert np.all(np.abs(a[both] - r[both]) <= 2 * tolerance(K, ex, den)[both]), i


def test_every_config(cuda, oracle_mod):
    import libthom_b200 as lt

    A, B, C0 = oracle_mod.make_half_problem(300, 520, 200, seed=7, lo=-1.0, hi=1.0)
    for cfg, name in enumerate(lt.hgemm_configs()):
        for beta in (-0.5, 0.0):
            C = run_tc(cuda, A, B, C0, 1.25, beta, config=cfg)
            assert check_against_exact(oracle_mod, C, A, B, C0, 1.25, beta) <= 1.0, name


@pytest.mark.parametrize("beta", [0.0, 2.0])
@pytest.mark.parametrize("M,N,K,offset", [(1, 1, 1, 0), (3, 5, 7, 0), (100, 64, 64, 0), (129, 65, 33, 0),
                                          (257, 300, 1000, 0), (520, 264, 72, 0), (136, 1032, 40, 0),
                                          (256, 256, 64, 1), (200, 136, 130, 1)])
def test_ragged_and_unaligned(cuda, oracle_mod, M, N, K, offset, beta):
    """Any M, N, K: partial tiles in every dimension (zero-filled TMA boxes, clipped TMA stores or
    masked stores), row pitches that are not multiples of 8 elements and 2-byte aligned pointers
    (packed operand copies, scalar epilogue). beta == 0 with an aligned C takes the staged TMA-store
    epilogue, beta != 0 the direct one."""
    A, B, C0 = oracle_mod.make_half_problem(M, N, K, seed=M + N + K, lo=-1.0, hi=1.0)
    C = run_tc(cuda, A, B, C0, 0.5, beta, offset=offset)
    assert check_against_exact(oracle_mod, C, A, B, C0, 0.5, beta) <= 1.0


def test_many_tiles_per_pair(cuda, oracle_mod):
    """Several tiles per CTA pair: the double-buffered TMEM accumulators cycle through both
    buffers and phases; checked on sampled rows of every 256-row block."""
    M, N, K = 4096, 4096, 192
    A, B, C0 = oracle_mod.make_half_problem(M, N, K, seed=11, lo=-1.0, hi=1.0)
    import libthom_b200 as lt

    rows = np.concatenate([np.arange(b, M, 256) for b in (0, 77, 128, 255)])
    for cfg in range(len(lt.hgemm_configs())):
        for beta in (0.0, 1.0):
            C = run_tc(cuda, A, B, C0, 1.0, beta, config=cfg)
            assert check_against_exact(oracle_mod, C, A, B, C0, 1.0, beta, rows=rows) <= 1.0


def test_k_zero_alpha_zero_beta_zero(cuda, oracle_mod):
    A, B, C0 = oracle_mod.make_half_problem(20, 30, 10, seed=1, lo=-2.0, hi=2.0)
    c0 = C0.view(np.float16).astype(np.float32)
    want = oracle_mod.half_bits(0.25 * c0)
    C = run_tc(cuda, np.zeros((20, 0), np.uint16), np.zeros((0, 30), np.uint16), C0, 2.0, 0.25)
    assert np.array_equal(C, want)
    C = run_tc(cuda, A, B, C0, 0.0, 0.25)
    assert np.array_equal(C, want)
    # beta == 0: C is not read, so NaN garbage in C does not leak into the result
    garbage = np.full((20, 30), 0x7E00, dtype=np.uint16)
    C = run_tc(cuda, A, B, garbage, 1.0, 0.0)
    assert np.all(np.isfinite(C.view(np.float16)))


def _reference_compare(gpu, cpu):
    """The reference's acceptance test (routines/hgemm/hgemm.cu:155-171): an entry differs when its
    relative error (against max(|ref|, 1e-3)) exceeds 1e-2 and its absolute error exceeds 1e-3."""
    g, c = gpu.view(np.float16).astype(np.float32), cpu.view(np.float16).astype(np.float32)
    diff = np.abs(g - c)
    rel = diff / np.maximum(np.abs(c), 1e-3)
    return int(np.sum((rel > 1e-2) & (diff > 1e-3)))


def test_reference_runner_setting_1024(cuda, oracle_mod):
    """The reference runner's own problem (1024^3, uniform (0, 1) inputs, alpha 1, beta 0,
    routines/hgemm/hgemm.cu:107-121): no entry fails the reference's acceptance test and every
    sampled entry is within the tolerance."""
    n = 1024
    A, B, C0 = oracle_mod.make_half_problem(n, n, n, seed=1234)
    C = run_tc(cuda, A, B, C0, 1.0, 0.0)
    rows = np.arange(0, n, 29)
    Cref = oracle_mod.hgemm_ref(A, B, C0, 1.0, 0.0, rows=rows)
    assert _reference_compare(C[rows], Cref) == 0
    assert check_against_exact(oracle_mod, C, A, B, C0, 1.0, 0.0, rows=rows) <= 1.0


@pytest.mark.slow
def test_full_size_8192_sampled_rows(cuda, oracle_mod):
    """8192^3 (the largest size of the reference's bench list, routines/hgemm/hgemm.cu:17-27) on
    sampled rows."""
    n = 8192
    A, B, C0 = oracle_mod.make_half_problem(n, n, n, seed=5, lo=-1.0, hi=1.0)
    C = run_tc(cuda, A, B, C0, 1.0, 0.5)
    rows = np.array([0, 255, 256, 4097, 8191])
    assert check_against_exact(oracle_mod, C, A, B, C0, 1.0, 0.5, rows=rows) <= 1.0


def test_agrees_with_cublas(cuda, oracle_mod):
    """cuBLAS with FP32 accumulation (the library's baseline call) obeys the same bound, and the two
    agree within twice of it; cuBLAS with the reference's FP16 accumulation passes the reference's
    acceptance test on the same problem."""
    import libthom_b200 as lt

    torch = cuda
    n = 2048
    A, B, C0 = oracle_mod.make_half_problem(n, n, n, seed=21)
    C = run_tc(torch, A, B, C0, 1.0, 0.0)
    dA, dB = dev(torch, A), dev(torch, B)
    dR = torch.zeros(n, n, dtype=torch.float16, device="cuda")
    lt.hgemm_cublas(dA, dB, dR, n, n, n, 1.0, 0.0, compute_f32=True)
    torch.cuda.synchronize()
    R = dR.view(torch.int16).cpu().numpy().view(np.uint16)
    rows = np.arange(0, n, 97)
    assert check_against_exact(oracle_mod, R, A, B, C0, 1.0, 0.0, rows=rows) <= 1.0
    ex, den = oracle_mod.hgemm_exact_rows(A, B, C0, 1.0, 0.0, rows=rows)
    a, r = C[rows].view(np.float16).astype(np.float64), R[rows].view(np.float16).astype(np.float64)
    assert np.all(np.abs(a - r) <= 2 * tolerance(n, ex, den))
    lt.hgemm_cublas(dA, dB, dR, n, n, n, 1.0, 0.0, compute_f32=False)
    torch.cuda.synchronize()
    R16 = dR.view(torch.int16).cpu().numpy().view(np.uint16)
    assert _reference_compare(R16[rows], oracle_mod.hgemm_ref(A, B, C0, 1.0, 0.0, rows=rows)) == 0


def test_reference_contract_wrapper_times(cuda, oracle_mod):
    import libthom_b200 as lt

    torch = cuda
    A, B, C0 = oracle_mod.make_half_problem(256, 256, 256, seed=2)
    dA, dB, dC = dev(torch, A), dev(torch, B), dev(torch, C0)
    assert lt.hgemm("tc100", dA, dB, dC, 256, 256, 256, 1.0, 0.0) > 0.0
    C = dC.view(torch.int16).cpu().numpy().view(np.uint16).reshape(256, 256)
    assert check_against_exact(oracle_mod, C, A, B, C0, 1.0, 0.0) <= 1.0
    assert lt.hgemm("cublas", dA, dB, dC, 256, 256, 256, 1.0, 0.0) > 0.0


def test_long_k(cuda, oracle_mod):
    """K = 65536 (1024 K blocks): FP32 accumulation over a long K stays within the bound, checked on
    rows from both CTAs of every pair tile."""
    M, N, K = 256, 264, 65536
    A, B, C0 = oracle_mod.make_half_problem(M, N, K, seed=31, lo=-1.0, hi=1.0)
    C = run_tc(cuda, A, B, C0, 1.0, 0.0)
    rows = np.array([0, 31, 64, 127, 128, 170, 255])
    assert check_against_exact(oracle_mod, C, A, B, C0, 1.0, 0.0, rows=rows) <= 1.0


def test_nonfinite_inputs_propagate_like_the_reference(cuda, oracle_mod):
    """An Inf or NaN in A or B makes exactly the outputs non-finite that the reference's check loop
    (routines/hgemm/hgemm.cu:135-149, restated) makes non-finite, with the same sign for Inf."""
    M, N, K = 70, 90, 200
    A, B, C0 = oracle_mod.make_half_problem(M, N, K, seed=17, lo=-1.0, hi=1.0)
    A[5, 17] = 0x7C00   # +Inf
    A[40, 3] = 0xFC00   # -Inf
    B[9, 61] = 0x7E00   # NaN
    for beta in (0.0, 0.5):
        C = run_tc(cuda, A, B, C0, 1.0, beta).view(np.float16)
        R = oracle_mod.hgemm_ref(A, B, C0, 1.0, beta).view(np.float16)
        assert np.array_equal(np.isnan(C), np.isnan(R))
        inf = np.isinf(R)
        assert np.array_equal(np.isinf(C), inf) and np.array_equal(np.sign(C[inf]), np.sign(R[inf]))
