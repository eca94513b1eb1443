"""ctypes bindings of the CPU oracle (oracle.c / oracle_blocked.c) and of oracle/_ref.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs
as the checker. The product library never uses it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_dgemm.so"
REF_FINAL_LIB = HERE / "_ref" / "libref_dgemm_final.so"
REF_HGEMM_LIB = HERE / "_ref" / "libref_hgemm.so"
REF_HGEMM_KERNELS_LIB = HERE / "_ref" / "libref_hgemm_kernels.so"

_c = ctypes
_vp, _i64, _i32, _f64, _u64 = _c.c_void_p, _c.c_int64, _c.c_int, _c.c_double, _c.c_uint64


# Where the reference project's sources are read from to build oracle/_ref: LIBTHOM_REFERENCE_SRC,
# else the checkout this build was developed against (absent on machines that only run the tests;
# there the prebuilt oracle/_ref files, or none, are used).
REFERENCE_SRC = os.environ.get("LIBTHOM_REFERENCE_SRC", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compiles liboracle.so, and oracle/_ref when the reference sources are present."""
    ref = REFERENCE_SRC if Path(REFERENCE_SRC, "routines").is_dir() else ""
    out = subprocess.run(["make", "-C", str(HERE), "all", f"REF={ref}"], stdout=subprocess.PIPE,
                         stderr=subprocess.STDOUT, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout)
    if not quiet:
        print(out.stdout)


_lib = None
_ref = None
_ref_final = None
_ref_hgemm = None
_ref_hgemm_kernels = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        L.oracle_mix64.restype = _u64
        L.oracle_mix64.argtypes = [_u64]
        L.oracle_bits.restype = _u64
        L.oracle_bits.argtypes = [_u64, _u64, _u64]
        L.oracle_uniform.restype = _f64
        L.oracle_uniform.argtypes = [_u64, _u64, _u64]
        L.oracle_fill.argtypes = [_vp, _i64, _u64, _u64, _i32]
        L.oracle_scale_rows.argtypes = [_vp, _i64, _i64, _u64, _u64, _i32]
        L.oracle_scale_cols.argtypes = [_vp, _i64, _i64, _u64, _u64, _i32]
        L.oracle_half_to_float.restype = _c.c_float
        L.oracle_half_to_float.argtypes = [_c.c_uint16]
        L.oracle_float_to_half.restype = _c.c_uint16
        L.oracle_float_to_half.argtypes = [_c.c_float]
        L.oracle_hgemm_ref.argtypes = [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _c.c_float, _c.c_float, _vp, _i64]
        L.oracle_hgemm_exact_rows.argtypes = [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _vp, _i64]
        L.oracle_dgemm_naive.argtypes = [_vp, _vp, _vp, _i32, _i32, _i32, _f64, _f64]
        L.oracle_dgemm_blocked.argtypes = [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _i32]
        L.oracle_dgemm_dot2_rows.argtypes = [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _vp, _i64, _i32]
        L.oracle_componentwise_error.argtypes = [_vp, _vp, _vp, _i64, _vp]
        L.oracle_ozaki_row_exponents.argtypes = [_vp, _i64, _i64, _vp]
        L.oracle_ozaki_col_exponents.argtypes = [_vp, _i64, _i64, _vp]
        L.oracle_ozaki_split_rows.argtypes = [_vp, _i64, _i64, _vp, _i32, _vp, _i64]
        L.oracle_ozaki_split_cols.argtypes = [_vp, _i64, _i64, _vp, _i32, _vp, _i64]
        L.oracle_ozaki_dgemm.argtypes = [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _i32, _i32]
        L.oracle_crt_shift.restype = _i32
        L.oracle_crt_shift.argtypes = [_vp, _i64, _i64, _i32, _i64]
        L.oracle_crt_row_shifts.argtypes = [_vp, _i64, _i64, _i32, _vp]
        L.oracle_crt_col_shifts.argtypes = [_vp, _i64, _i64, _i32, _vp]
        L.oracle_crt_split_rows.argtypes = [_vp, _i64, _i64, _vp, _i32, _vp, _vp, _i64]
        L.oracle_crt_split_cols.argtypes = [_vp, _i64, _i64, _vp, _i32, _vp, _vp, _i64]
        L.oracle_crt_dgemm.argtypes = [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _i32, _i32, _i32, _i32, _i32,
                                       _vp, _vp, _vp, _f64, _f64, _i32]
        L.oracle_ozaki_analytic_slices.restype = _i32
        L.oracle_ozaki_analytic_slices.argtypes = [_f64, _i32]
        L.oracle_max_gap.restype = _i32
        L.oracle_max_gap.argtypes = [_vp, _i64, _i64, _i32]
        L.oracle_features.argtypes = [_vp, _vp, _i64, _i64, _i64, _f64, _vp]
        L.oracle_mlp_forward.argtypes = [_vp, _vp, _i32, _vp]
        L.oracle_mlp_backward.restype = _f64
        L.oracle_mlp_backward.argtypes = [_vp, _vp, _vp, _i32, _vp]
        _lib = L
    return _lib


def ref_lib() -> ctypes.CDLL | None:
    """The reference's own host check loop (routines/dgemm/dgemm.cpp:122-133), if built here."""
    global _ref
    if _ref is None and REF_LIB.exists():
        R = ctypes.CDLL(str(REF_LIB))
        R.ref_dgemm_host.argtypes = [_vp, _vp, _vp, _i32, _i32, _i32, _f64, _f64]
        _ref = R
    return _ref


def ref_final_lib() -> ctypes.CDLL | None:
    """The reference's dgemm_final CUDA kernel (routines/dgemm/dgemm_final.cu) built for sm_100a,
    if built here: ref_dgemm_final(A, B, C, M, N, K, alpha, beta) on device pointers, returning
    the milliseconds its own CUDA events measured."""
    global _ref_final
    if _ref_final is None and REF_FINAL_LIB.exists():
        R = ctypes.CDLL(str(REF_FINAL_LIB))
        R.ref_dgemm_final.restype = ctypes.c_float
        R.ref_dgemm_final.argtypes = [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, _f64, _f64]
        _ref_final = R
    return _ref_final


def ref_hgemm_lib() -> ctypes.CDLL | None:
    """The reference's own HGEMM host check (routines/hgemm/hgemm.cu:135-149), if built here:
    ref_hgemm_host(A, B, C, M, N, K, alpha_bits, beta_bits) overwrites C (FP16 bit patterns)."""
    global _ref_hgemm
    if _ref_hgemm is None and REF_HGEMM_LIB.exists():
        R = ctypes.CDLL(str(REF_HGEMM_LIB))
        R.ref_hgemm_host.argtypes = [_vp, _vp, _vp, _i32, _i32, _i32, _c.c_uint16, _c.c_uint16]
        _ref_hgemm = R
    return _ref_hgemm


def ref_hgemm_kernels_lib() -> ctypes.CDLL | None:
    """The reference's HGEMM CUDA kernels hgemm_final and hgemm_better_reuse built for sm_100a, if
    built here: ref_hgemm_final / ref_hgemm_better_reuse(A, B, C, M, N, K, alpha_bits, beta_bits)
    on device pointers, returning the milliseconds of their own CUDA events."""
    global _ref_hgemm_kernels
    if _ref_hgemm_kernels is None and REF_HGEMM_KERNELS_LIB.exists():
        R = ctypes.CDLL(str(REF_HGEMM_KERNELS_LIB))
        for name in ("ref_hgemm_final", "ref_hgemm_better_reuse"):
            f = getattr(R, name)
            f.restype = ctypes.c_float
            f.argtypes = [_vp, _vp, _vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, _c.c_uint16, _c.c_uint16]
        _ref_hgemm_kernels = R
    return _ref_hgemm_kernels


def half_bits(x) -> np.ndarray:
    """FP16 bit patterns (uint16) of an array of numbers (numpy's float16 rounding, ties to even)."""
    return np.array(x, dtype=np.float16, order="C").view(np.uint16)


def make_half_problem(M: int, N: int, K: int, seed: int = 1234, lo: float = 0.0, hi: float = 1.0):
    """FP16 inputs A (M x K), B (K x N), C0 (M x N) as uint16 bit patterns, uniform in [lo, hi) then
    rounded to FP16 (the reference's fill is cuRAND uniform (0, 1] rounded to FP16,
    routines/hgemm/hgemm.cu:107-119)."""
    rng = np.random.default_rng(seed)
    A = half_bits(rng.uniform(lo, hi, size=(M, K)))
    B = half_bits(rng.uniform(lo, hi, size=(K, N)))
    C0 = half_bits(rng.uniform(lo, hi, size=(M, N)))
    return A, B, C0


def hgemm_ref(A, B, C0, alpha: float, beta: float, rows=None) -> np.ndarray:
    """The reference's HGEMM host check restated (oracle_hgemm_ref) on uint16 bit patterns; the
    selected rows (all by default) of C as uint16."""
    M, K = A.shape
    N = B.shape[1]
    A, B, C0 = (np.ascontiguousarray(x, dtype=np.uint16) for x in (A, B, C0))
    if rows is None:
        out = np.empty((M, N), dtype=np.uint16)
        lib().oracle_hgemm_ref(_p(A), _p(B), _p(C0), _p(out), M, N, K, alpha, beta, None, 0)
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.empty((len(rows), N), dtype=np.uint16)
        lib().oracle_hgemm_ref(_p(A), _p(B), _p(C0), _p(out), M, N, K, alpha, beta, _p(rows), len(rows))
    return out


def hgemm_exact_rows(A, B, C0, alpha: float, beta: float, rows=None):
    """float64 value and componentwise denominator |alpha| sum |a||b| + |beta||c| of the selected
    rows of alpha*A*B + beta*C0."""
    M, K = A.shape
    N = B.shape[1]
    A, B, C0 = (np.ascontiguousarray(x, dtype=np.uint16) for x in (A, B, C0))
    rows = np.arange(M, dtype=np.int64) if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
    ex = np.empty((len(rows), N))
    den = np.empty((len(rows), N))
    lib().oracle_hgemm_exact_rows(_p(A), _p(B), _p(C0), _p(ex), _p(den), M, N, K, alpha, beta, _p(rows), len(rows))
    return ex, den


def hgemm_ref_loop(A, B, C0, alpha_bits: int, beta_bits: int) -> np.ndarray | None:
    """C from the reference's own compiled host check, or None if oracle/_ref is not built."""
    R = ref_hgemm_lib()
    if R is None:
        return None
    M, K = A.shape
    N = B.shape[1]
    C = np.ascontiguousarray(C0, dtype=np.uint16).copy()
    A, B = (np.ascontiguousarray(x, dtype=np.uint16) for x in (A, B))
    R.ref_hgemm_host(_p(A), _p(B), _p(C), M, N, K, alpha_bits, beta_bits)
    return C


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def nthreads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


# ---- generator ---------------------------------------------------------------------------------
def fill(rows: int, cols: int, stream: int, phi: int = 0, seed: int = 1234) -> np.ndarray:
    x = np.empty((rows, cols), dtype=np.float64)
    lib().oracle_fill(_p(x), rows * cols, seed, stream, phi)
    return x


def scale_rows(x: np.ndarray, seed: int, stream: int, smax: int) -> None:
    lib().oracle_scale_rows(_p(x), x.shape[0], x.shape[1], seed, stream, smax)


def scale_cols(x: np.ndarray, seed: int, stream: int, smax: int) -> None:
    lib().oracle_scale_cols(_p(x), x.shape[0], x.shape[1], seed, stream, smax)


def make_problem(M: int, N: int, K: int, phi: int = 0, seed: int = 1234, smax: int = 0):
    """A (stream 1), B (stream 2), C0 (stream 3); rows of A / columns of B scaled by 2^s with
    s ~ U{-smax..smax} (streams 4, 5) when smax > 0."""
    A = fill(M, K, 1, phi, seed)
    B = fill(K, N, 2, phi, seed)
    C0 = fill(M, N, 3, phi, seed)
    if smax > 0:
        scale_rows(A, seed, 4, smax)
        scale_cols(B, seed, 5, smax)
    return A, B, C0


# ---- GEMM oracles ------------------------------------------------------------------------------
def dgemm_naive(A, B, C0, alpha, beta) -> np.ndarray:
    M, K = A.shape
    N = B.shape[1]
    C = np.ascontiguousarray(C0).copy()
    lib().oracle_dgemm_naive(_p(A), _p(B), _p(C), M, N, K, alpha, beta)
    return C


def dgemm_ref(A, B, C0, alpha, beta) -> np.ndarray | None:
    R = ref_lib()
    if R is None:
        return None
    M, K = A.shape
    N = B.shape[1]
    C = np.ascontiguousarray(C0).copy()
    R.ref_dgemm_host(_p(A), _p(B), _p(C), M, N, K, alpha, beta)
    return C


def dgemm_blocked(A, B, C0, alpha, beta, threads: int | None = None) -> np.ndarray:
    M, K = A.shape
    N = B.shape[1]
    C = np.ascontiguousarray(C0).copy()
    lib().oracle_dgemm_blocked(_p(A), _p(B), _p(C), M, N, K, alpha, beta, threads or nthreads())
    return C


def dot2_rows(A, B, C0, alpha, beta, rows=None, threads: int | None = None):
    """Near-exact C and the componentwise denominator on the listed rows."""
    M, K = A.shape
    N = B.shape[1]
    rows = np.arange(M, dtype=np.int64) if rows is None else np.ascontiguousarray(rows, dtype=np.int64)
    Cref = np.empty((len(rows), N))
    den = np.empty((len(rows), N))
    c0 = np.ascontiguousarray(C0) if C0 is not None else np.zeros((M, N))
    lib().oracle_dgemm_dot2_rows(_p(A), _p(B), _p(c0), _p(Cref), _p(den), M, N, K, alpha, beta, _p(rows),
                                 len(rows), threads or nthreads())
    return Cref, den


def componentwise_error(C, Cref, den):
    """(max, median, mean, non-finite mismatches) of |C - Cref| / den."""
    out = np.zeros(4)
    C = np.ascontiguousarray(C, dtype=np.float64)
    lib().oracle_componentwise_error(_p(C), _p(np.ascontiguousarray(Cref)), _p(np.ascontiguousarray(den)), C.size,
                                     _p(out))
    return tuple(out)


# ---- Ozaki restatement -------------------------------------------------------------------------
def ozaki_dgemm(A, B, C0, alpha, beta, s, threads: int | None = None) -> np.ndarray:
    M, K = A.shape
    N = B.shape[1]
    C = np.ascontiguousarray(C0).copy()
    lib().oracle_ozaki_dgemm(_p(A), _p(B), _p(C), M, N, K, alpha, beta, s, threads or nthreads())
    return C


def ozaki_split(A, B, s):
    """(sigma, tau, A slices [s][M][Kp], B slices [s][N][Kp])."""
    M, K = A.shape
    N = B.shape[1]
    Kp = (max(K, 1) + 31) // 32 * 32
    sigma = np.empty(M, dtype=np.int32)
    tau = np.empty(N, dtype=np.int32)
    sa = np.empty((s, M, Kp), dtype=np.int8)
    sb = np.empty((s, N, Kp), dtype=np.int8)
    L = lib()
    L.oracle_ozaki_row_exponents(_p(A), M, K, _p(sigma))
    L.oracle_ozaki_col_exponents(_p(B), K, N, _p(tau))
    L.oracle_ozaki_split_rows(_p(A), M, K, _p(sigma), s, _p(sa), Kp)
    L.oracle_ozaki_split_cols(_p(B), K, N, _p(tau), s, _p(sb), Kp)
    return sigma, tau, sa, sb


# ---- Ozaki scheme II (CRT form) restatement -----------------------------------------------------
# Pairwise-coprime moduli no larger than 256 (so every symmetric residue is one signed byte), largest
# first; a CRT-form DGEMM with n moduli uses the first n.
CRT_MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181, 179, 173)
CRT_MIN, CRT_MAX = 8, 20


def crt_norm_bits(Mp: int) -> tuple[int, int]:
    """(ta, tb): the rows of A are scaled to 2-norm at most 2^ta and the columns of B to at most 2^tb,
    with ta + tb = Tc the largest integer such that 2^Tc <= Mprod (1 - 2^-20) / 2 (each at most 62):
    then |sum_k V W| <= |V|_2 |W|_2 < Mprod / 2 by the Cauchy-Schwarz inequality."""
    Tc = (Mp * (2 ** 20 - 1) // 2 ** 21).bit_length() - 1
    return min(62, Tc // 2), min(62, Tc - Tc // 2)


def crt_constants(n: int) -> dict:
    """Constants of the CRT form with n moduli, by exact integer arithmetic: Mprod, the limb width w
    and count nl, the limbs P[l][k] of the CRT basis P_l = (Mprod/m_l) * ((Mprod/m_l)^-1 mod m_l), the
    limbs of Mprod, f_hi / f_lo = 2^(w k) / Mprod_d (Mprod_d = the limbs summed by Horner in double),
    and the norm bounds ta, tb (crt_norm_bits)."""
    assert CRT_MIN <= n <= CRT_MAX
    mods = CRT_MODULI[:n]
    Mp = 1
    for m in mods:
        Mp *= m
    w = 42 if n <= 16 else 41
    nl = -(-Mp.bit_length() // w)
    mask = (1 << w) - 1
    P = []
    for m in mods:
        Ml = Mp // m
        P.append(Ml * pow(Ml % m, -1, m))
    Pl = np.array([[float((p >> (w * k)) & mask) for k in range(nl)] for p in P], dtype=np.float64)
    Mk = np.array([float((Mp >> (w * k)) & mask) for k in range(nl)], dtype=np.float64)
    md = float(Mk[nl - 1])
    for k in range(nl - 2, -1, -1):
        md = md * 2.0 ** w + float(Mk[k])  # exact scaling, one rounding per step (= fma(md, 2^w, M_k))
    ta, tb = crt_norm_bits(Mp)
    return {"n": n, "mods": np.array(mods, dtype=np.int32), "Mprod": Mp, "w": w, "nl": nl, "P": Pl, "Mk": Mk,
            "f_hi": 2.0 ** (w * (nl - 1)) / md, "f_lo": 2.0 ** (w * (nl - 2)) / md, "ta": ta, "tb": tb}


def crt_dgemm(A, B, C0, alpha, beta, n, threads: int | None = None) -> np.ndarray:
    """The CRT form restated (oracle_crt_dgemm) with n moduli."""
    M, K = A.shape
    N = B.shape[1]
    c = crt_constants(n)
    C = np.ascontiguousarray(C0).copy()
    P = np.ascontiguousarray(c["P"])
    lib().oracle_crt_dgemm(_p(np.ascontiguousarray(A)), _p(np.ascontiguousarray(B)), _p(C), M, N, K, alpha, beta, n,
                           c["nl"], c["w"], c["ta"], c["tb"], _p(c["mods"]), _p(P), _p(c["Mk"]), c["f_hi"], c["f_lo"],
                           threads or nthreads())
    return C


def crt_shifts(A, B, n):
    """(row shifts of A, column shifts of B) of the CRT form with n moduli (oracle_crt_shift)."""
    M, K = A.shape
    N = B.shape[1]
    c = crt_constants(n)
    sa = np.empty(M, dtype=np.int32)
    sb = np.empty(N, dtype=np.int32)
    A, B = np.ascontiguousarray(A), np.ascontiguousarray(B)
    lib().oracle_crt_row_shifts(_p(A), M, K, c["ta"], _p(sa))
    lib().oracle_crt_col_shifts(_p(B), K, N, c["tb"], _p(sb))
    return sa, sb


def crt_split(A, B, n):
    """(row shifts, column shifts, residues of A [n][M][K], residues of B transposed [n][N][K]) of the
    CRT form."""
    M, K = A.shape
    N = B.shape[1]
    c = crt_constants(n)
    Kp = max(K, 1)
    sa, sb = crt_shifts(A, B, n)
    ra = np.empty((n, M, Kp), dtype=np.int8)
    rb = np.empty((n, N, Kp), dtype=np.int8)
    L = lib()
    A, B = np.ascontiguousarray(A), np.ascontiguousarray(B)
    L.oracle_crt_split_rows(_p(A), M, K, _p(sa), n, _p(c["mods"]), _p(ra), Kp)
    L.oracle_crt_split_cols(_p(B), K, N, _p(sb), n, _p(c["mods"]), _p(rb), Kp)
    return sa, sb, ra, rb


def analytic_slices(tol: float, gap_bits: int) -> int:
    return int(lib().oracle_ozaki_analytic_slices(tol, gap_bits))


def gap_bits(A, B) -> int:
    """Largest exponent gap within a row of A plus the largest within a column of B."""
    L = lib()
    return int(L.oracle_max_gap(_p(A), A.shape[0], A.shape[1], 1)) + int(L.oracle_max_gap(_p(B), B.shape[0], B.shape[1], 0))


# ---- selector restatements ---------------------------------------------------------------------
SEL_F, SEL_H, SEL_C = 34, 64, 8
SEL_P = SEL_F * SEL_H + SEL_H + SEL_H * SEL_H + SEL_H + SEL_H * SEL_C + SEL_C


def features(A, B, tol: float) -> np.ndarray:
    M, K = A.shape
    N = B.shape[1]
    f = np.empty(SEL_F, dtype=np.float32)
    lib().oracle_features(_p(A), _p(B), M, N, K, tol, _p(f))
    return f


def mlp_forward(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty((x.shape[0], SEL_C), dtype=np.float32)
    lib().oracle_mlp_forward(_p(np.ascontiguousarray(params, dtype=np.float32)), _p(x), x.shape[0], _p(out))
    return out


def mlp_backward(params: np.ndarray, x: np.ndarray, labels: np.ndarray):
    """(mean loss, mean gradient) in double precision."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(labels, dtype=np.int32)
    g = np.empty(SEL_P, dtype=np.float64)
    loss = lib().oracle_mlp_backward(_p(np.ascontiguousarray(params, dtype=np.float32)), _p(x), _p(y), x.shape[0], _p(g))
    return float(loss), g
