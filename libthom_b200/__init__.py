"""libthom_b200 — sm_100a (B200) DGEMM for libthom's `dgemm` routine.

The product is the C-ABI shared library ``liblibthom_dgemm.so`` built from ``csrc/`` (declared in
``include/libthom_dgemm.h``). This module only loads it with ctypes and gives Python callers the
same entry points; it never computes anything itself. If the library is missing or no sm_100 GPU
is present, calls raise — there is no CPU fallback.

Implementation registry (the reference's ``dgemmImpls``, routines/dgemm/dgemm.cpp:36-68):
``tc100`` (native FP64 tensor cores), ``ozaki3`` .. ``ozaki10`` (INT8 Ozaki slices),
``ozaki_auto`` (learned slice selector), ``auto`` (native FP64 or Ozaki, whichever is faster for the
shape) and ``cublas_tc`` (the reference's cuBLAS baseline).
"""
from __future__ import annotations

import ctypes
import os
import struct
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblibthom_dgemm.so"

LT_OK = 0
LT_ERR_INVALID_ARGUMENT = 1
LT_ERR_UNALIGNED = 2
LT_ERR_CUDA = 3
LT_ERR_NO_MEMORY = 4
LT_ERR_DEVICE_TIMEOUT = 5
LT_ERR_UNSUPPORTED = 6
LT_ERR_NOT_FOUND = 7
LT_OZAKI_MAX_SLICES = 12
LT_OZAKI_CRT_MIN_MODULI = 8
LT_OZAKI_CRT_MAX_MODULI = 20
LT_FORM_FP64 = 0
LT_FORM_OZAKI = 1
LT_PEAK_FP64_MMA = 0
LT_PEAK_INT8_MMA_N128 = 1
LT_PEAK_INT8_MMA_N256 = 2
LT_PEAK_INT8_MMA_PAIR = 3
LT_PEAK_SUSTAINED = 0x10
LT_SEL_FEATURES = 34
LT_SEL_HIDDEN = 64
LT_SEL_CLASSES = 8
LT_SEL_PARAMS = (LT_SEL_FEATURES * LT_SEL_HIDDEN + LT_SEL_HIDDEN + LT_SEL_HIDDEN * LT_SEL_HIDDEN +
                 LT_SEL_HIDDEN + LT_SEL_HIDDEN * LT_SEL_CLASSES + LT_SEL_CLASSES)

IMPLS = (["tc100"] + [f"ozaki{s}" for s in range(3, 11)] + ["ozaki_auto", "auto", "cublas_tc"]
         + [f"ozaki_crt{n}" for n in range(14, 19)])

_c = ctypes
_vp, _i64, _i32, _f64, _f32, _sz = _c.c_void_p, _c.c_int64, _c.c_int, _c.c_double, _c.c_float, _c.c_size_t
_u64 = _c.c_uint64


class LtError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"libthom_dgemm error {code}: {message}")
        self.code = code


class GemmProblem(ctypes.Structure):
    """lt_gemm_problem (include/libthom_dgemm.h)."""
    _fields_ = [("M", _i64), ("N", _i64), ("K", _i64), ("A", _vp), ("B", _vp), ("C", _vp),
                ("alpha", _f64), ("beta", _f64)]


class TuneEntry(ctypes.Structure):
    _fields_ = [("config", _i32), ("ms", _f32), ("max_rel_err", _f32)]


# name -> (restype, argtypes)
_GEMM = [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64]
_REF = [_vp, _vp, _vp, _sz, _sz, _sz, _f64, _f64]
_HGEMM = [_vp, _vp, _vp, _i64, _i64, _i64, _f32, _f32]
_HREF = [_vp, _vp, _vp, _sz, _sz, _sz, _c.c_uint16, _c.c_uint16]
SIGNATURES = {
    "lt_get_last_error": (_i32, []),
    "lt_error_string": (_c.c_char_p, [_i32]),
    "lt_last_error_message": (_c.c_char_p, []),
    "lt_check_device_status": (_i32, []),
    "lt_selftest_wait_timeout": (_i32, [_f64, _vp]),
    "lt_version": (_i32, []),
    "dgemm_tc100": (_f32, _REF),
    "dgemm_ozaki3": (_f32, _REF), "dgemm_ozaki4": (_f32, _REF), "dgemm_ozaki5": (_f32, _REF),
    "dgemm_ozaki6": (_f32, _REF), "dgemm_ozaki7": (_f32, _REF), "dgemm_ozaki8": (_f32, _REF),
    "dgemm_ozaki9": (_f32, _REF), "dgemm_ozaki10": (_f32, _REF),
    "dgemm_ozaki_auto": (_f32, _REF),
    "dgemm_auto": (_f32, _REF),
    "lt_dgemm_auto": (_i32, _GEMM + [_c.POINTER(_i32), _c.POINTER(_i32), _vp]),
    "lt_dgemm_estimate_ms": (_f64, [_i32, _i64, _i64, _i64, _i32]),
    "dgemm_cublas_tc": (_f32, _REF),
    "lt_dgemm_fp64": (_i32, _GEMM + [_vp]),
    "lt_dgemm_fp64_config": (_i32, _GEMM + [_i32, _vp]),
    "lt_fp64_num_configs": (_i32, []),
    "lt_fp64_config_name": (_c.c_char_p, [_i32]),
    "lt_dgemm_ozaki": (_i32, _GEMM + [_i32, _vp]),
    "lt_ozaki_workspace_size": (_sz, [_i64, _i64, _i64, _i32]),
    "lt_dgemm_ozaki_ws": (_i32, _GEMM + [_i32, _vp, _sz, _vp]),
    "lt_ozaki_split": (_i32, [_vp, _vp, _i64, _i64, _i64, _i32, _vp, _sz, _vp]),
    "lt_ozaki_product": (_i32, [_vp, _i64, _i64, _i64, _f64, _f64, _i32, _vp, _sz, _vp]),
    "lt_dgemm_cublas": (_i32, _GEMM + [_vp]),
    "lt_dgemm_ozaki_noalloc": (_i32, _GEMM + [_i32, _vp]),
    "lt_dgemm_ozaki_crt": (_i32, _GEMM + [_i32, _vp]),
    "lt_ozaki_crt_workspace_size": (_sz, [_i64, _i64, _i64, _i32]),
    "lt_dgemm_ozaki_crt_ws": (_i32, _GEMM + [_i32, _vp, _sz, _vp]),
    "lt_ozaki_crt_split": (_i32, [_vp, _vp, _i64, _i64, _i64, _i32, _vp, _sz, _vp]),
    "lt_ozaki_crt_product": (_i32, [_vp, _i64, _i64, _i64, _f64, _f64, _i32, _vp, _sz, _vp]),
    "lt_dgemm_ozaki_crt_host": (_i32, _GEMM + [_i32, _vp]),
    "lt_ozaki_crt_multiply": (_i32, [_i64, _i64, _i64, _i32, _vp, _sz, _vp]),
    "lt_ozaki_crt_reconstruct": (_i32, [_vp, _i64, _i64, _i64, _f64, _f64, _i32, _vp, _sz, _vp]),
    "lt_ozaki_crt_info": (_i32, [_i32, _c.POINTER(_i32), _c.POINTER(_i32), _c.POINTER(_i32)]),
    "dgemm_ozaki_crt14": (_f32, _REF), "dgemm_ozaki_crt15": (_f32, _REF), "dgemm_ozaki_crt16": (_f32, _REF),
    "dgemm_ozaki_crt17": (_f32, _REF), "dgemm_ozaki_crt18": (_f32, _REF),
    "lt_selftest_wait_timeout_noalloc": (_i32, [_f64, _vp]),
    "lt_grouped_plan_create": (_i32, [_vp, _i32, _i32, _i32, _c.POINTER(_vp)]),
    "lt_grouped_plan_run": (_i32, [_vp, _vp]),
    "lt_grouped_plan_run_graph": (_i32, [_vp, _vp]),
    "lt_grouped_plan_info": (_i32, [_vp, _c.POINTER(_i64), _c.POINTER(_f64)]),
    "lt_grouped_plan_destroy": (None, [_vp]),
    "lt_grouped_plan_tune": (_i32, [_vp, _i32, _c.POINTER(_f32)]),
    "lt_grouped_plan_config": (_i32, [_vp, _c.c_char_p, _i32]),
    "lt_dgemm_grouped": (_i32, [_vp, _i32, _i32, _i32, _vp]),
    "lt_tune_fp64": (_i32, [_i64, _i64, _i64, _i32, _c.POINTER(TuneEntry)]),
    "lt_tuner_save": (_i32, [_c.c_char_p]),
    "lt_tuner_load": (_i32, [_c.c_char_p]),
    "lt_tuner_lookup": (_i32, [_i64, _i64, _i64]),
    "lt_ozaki_features": (_i32, [_vp, _vp, _i64, _i64, _i64, _f64, _vp, _vp]),
    "lt_mlp_forward": (_i32, [_vp, _vp, _i32, _vp, _vp]),
    "lt_mlp_train_step": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp, _i32, _f32, _i32, _vp, _vp]),
    "lt_mlp_backward": (_i32, [_vp, _vp, _vp, _i32, _vp, _vp, _vp]),
    "lt_selector_set_params": (_i32, [_vp]),
    "lt_set_ozaki_tolerance": (None, [_f64]),
    "lt_ozaki_analytic_slices": (_i32, [_f64, _i32]),
    "lt_ozaki_gap_bits": (_i32, [_vp, _vp, _i64, _i64, _i64, _c.POINTER(_i32), _vp]),
    "lt_ozaki_select_slices": (_i32, [_vp, _vp, _i64, _i64, _i64, _f64, _c.POINTER(_i32), _vp]),
    "lt_ozaki_auto_plan_create": (_i32, [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _f64, _i32, _c.POINTER(_vp)]),
    "lt_ozaki_auto_plan_run": (_i32, [_vp, _vp]),
    "lt_ozaki_auto_plan_choice": (_i32, [_vp, _c.POINTER(_i32), _c.POINTER(_i32)]),
    "lt_ozaki_auto_plan_destroy": (None, [_vp]),
    "lt_ozaki_select_info": (_i32, [_vp, _vp, _i64, _i64, _i64, _f64, _c.POINTER(_i32), _c.POINTER(_i32),
                                    _c.POINTER(_i32), _vp]),
    "lt_fill": (_i32, [_vp, _i64, _u64, _u64, _i32, _vp]),
    "lt_scale_rows": (_i32, [_vp, _i64, _i64, _u64, _u64, _i32, _vp]),
    "lt_scale_cols": (_i32, [_vp, _i64, _i64, _u64, _u64, _i32, _vp]),
    "lt_componentwise_error": (_i32, [_vp, _vp, _vp, _i64, _f64, _c.POINTER(_f64), _vp]),
    "lt_abs_denominator": (_i32, [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _vp]),
    "lt_flush_l2": (_i32, [_vp]),
    "lt_measure_peak": (_i32, [_i32, _c.POINTER(_f64), _vp]),
    "lt_grouped_num_configs": (_i32, []),
    "lt_grouped_config_name": (_c.c_char_p, [_i32]),
    "lt_grouped_plan_set_fp64": (_i32, [_vp, _i32, _i32, _i64]),
    "lt_dgemm_ozaki_host": (_i32, [_vp, _vp, _vp, _i64, _i64, _i64, _f64, _f64, _i32, _vp]),
    "lt_dgemm_ex": (_i32, [_i32, _c.c_char, _c.c_char, _i64, _i64, _i64, _f64, _vp, _i64, _vp, _i64, _f64, _vp, _i64,
                           _i32, _vp]),
    "lt_dot2_rows": (_i32, [_vp, _vp, _vp, _f64, _f64, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _vp]),
    # libthom_hgemm.h
    "hgemm_tc100": (_f32, _HREF),
    "hgemm_cublas": (_f32, _HREF),
    "lt_hgemm": (_i32, _HGEMM + [_vp]),
    "lt_hgemm_config": (_i32, _HGEMM + [_i32, _vp]),
    "lt_hgemm_num_configs": (_i32, []),
    "lt_hgemm_config_name": (_c.c_char_p, [_i32]),
    "lt_hgemm_default_config": (_i32, [_i64, _i64, _i64]),
    "lt_hgemm_cublas": (_i32, _HGEMM + [_i32, _vp]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library. Raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m libthom_b200.build` "
                               "(the DGEMM has no CPU fallback)")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != LT_OK:
        msg = lib().lt_last_error_message()
        raise LtError(rc, (msg or b"").decode(errors="replace"))


def _ptr(x) -> int:
    """Device pointer of a torch tensor, or an int pointer as is."""
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(stream) -> int | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def dgemm(impl: str, A, B, C, M: int, N: int, K: int, alpha: float = 1.0, beta: float = 0.0) -> float:
    """Reference-contract call (routines/dgemm/dgemm.h:9): synchronous, returns elapsed ms."""
    if impl not in IMPLS:
        raise KeyError(f"unknown implementation {impl!r}; available: {' '.join(IMPLS)}")
    fn = getattr(lib(), "dgemm_" + impl)
    ms = fn(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta)
    check(lib().lt_get_last_error())
    return ms


def dgemm_fp64(A, B, C, M, N, K, alpha=1.0, beta=0.0, stream=None, config: int = -1) -> None:
    if config < 0:
        check(lib().lt_dgemm_fp64(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, _stream(stream)))
    else:
        check(lib().lt_dgemm_fp64_config(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, config,
                                         _stream(stream)))


LT_AUTO_PLAN_OZAKI, LT_AUTO_PLAN_ANY_FORM = 0, 1


class OzakiAutoPlan:
    """lt_ozaki_auto_plan: slice selection and the slice form (or, with forms=LT_AUTO_PLAN_ANY_FORM,
    native FP64 where the cost model prefers it) in one CUDA graph with the choice made on the device.
    Holds the tensors' pointers; run() replays the graph on `stream` without host synchronisation."""

    def __init__(self, A, B, C, M, N, K, alpha, beta, tol, forms=LT_AUTO_PLAN_OZAKI):
        self._h = ctypes.c_void_p()
        self._keep = (A, B, C)
        check(lib().lt_ozaki_auto_plan_create(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, tol, forms,
                                              ctypes.byref(self._h)))

    def run(self, stream=None) -> None:
        check(lib().lt_ozaki_auto_plan_run(self._h, _stream(stream)))

    def choice(self) -> tuple[int, bool]:
        """(slice count, learned?) of the last run; slice count 0: native FP64 ran (synchronous)."""
        s, learned = ctypes.c_int(), ctypes.c_int()
        check(lib().lt_ozaki_auto_plan_choice(self._h, ctypes.byref(s), ctypes.byref(learned)))
        return s.value, bool(learned.value)

    def close(self) -> None:
        if self._h:
            lib().lt_ozaki_auto_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dgemm_ozaki(A, B, C, M, N, K, alpha=1.0, beta=0.0, slices=8, stream=None, workspace=None) -> None:
    if workspace is None:
        check(lib().lt_dgemm_ozaki(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, slices, _stream(stream)))
    else:
        check(lib().lt_dgemm_ozaki_ws(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, slices,
                                      _ptr(workspace), workspace.numel() * workspace.element_size(),
                                      _stream(stream)))


def dgemm_ozaki_crt(A, B, C, M, N, K, alpha=1.0, beta=0.0, moduli=15, stream=None, workspace=None) -> None:
    """CRT form (Ozaki scheme II) with `moduli` INT8 products (lt_dgemm_ozaki_crt / _ws)."""
    if workspace is None:
        check(lib().lt_dgemm_ozaki_crt(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, moduli, _stream(stream)))
    else:
        check(lib().lt_dgemm_ozaki_crt_ws(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, moduli, _ptr(workspace),
                                          workspace.numel() * workspace.element_size(), _stream(stream)))


def ozaki_crt_split(A, B, M, N, K, moduli, workspace, stream=None) -> None:
    check(lib().lt_ozaki_crt_split(_ptr(A), _ptr(B), M, N, K, moduli, _ptr(workspace),
                                   workspace.numel() * workspace.element_size(), _stream(stream)))


def ozaki_crt_product(C, M, N, K, alpha, beta, moduli, workspace, stream=None) -> None:
    check(lib().lt_ozaki_crt_product(_ptr(C), M, N, K, alpha, beta, moduli, _ptr(workspace),
                                     workspace.numel() * workspace.element_size(), _stream(stream)))


def dgemm_ozaki_crt_host(A, B, C, M, N, K, alpha=1.0, beta=0.0, moduli=15, stream=None) -> None:
    """CRT form on host (CPU) tensors or arrays, pipelined through the GPU (lt_dgemm_ozaki_crt_host).
    C holds C0 on entry and the result on return."""
    check(lib().lt_dgemm_ozaki_crt_host(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, moduli, _stream(stream)))


def ozaki_crt_multiply(M, N, K, moduli, workspace, stream=None) -> None:
    check(lib().lt_ozaki_crt_multiply(M, N, K, moduli, _ptr(workspace), workspace.numel() * workspace.element_size(),
                                      _stream(stream)))


def ozaki_crt_reconstruct(C, M, N, K, alpha, beta, moduli, workspace, stream=None) -> None:
    check(lib().lt_ozaki_crt_reconstruct(_ptr(C), M, N, K, alpha, beta, moduli, _ptr(workspace),
                                         workspace.numel() * workspace.element_size(), _stream(stream)))


def ozaki_crt_workspace_size(M, N, K, moduli) -> int:
    return int(lib().lt_ozaki_crt_workspace_size(M, N, K, moduli))


def ozaki_crt_info(moduli: int) -> tuple[int, int, list[int]]:
    """(ta, tb, moduli list) of the CRT form (host arithmetic): the rows of A are scaled to 2-norm at
    most 2^ta, the columns of B to at most 2^tb."""
    ta, tb = ctypes.c_int(), ctypes.c_int()
    mods = (ctypes.c_int * moduli)()
    check(lib().lt_ozaki_crt_info(moduli, ctypes.byref(ta), ctypes.byref(tb), mods))
    return ta.value, tb.value, list(mods)


def ozaki_split(A, B, M, N, K, slices, workspace, stream=None) -> None:
    check(lib().lt_ozaki_split(_ptr(A), _ptr(B), M, N, K, slices, _ptr(workspace),
                               workspace.numel() * workspace.element_size(), _stream(stream)))


def ozaki_product(C, M, N, K, alpha, beta, slices, workspace, stream=None) -> None:
    check(lib().lt_ozaki_product(_ptr(C), M, N, K, alpha, beta, slices, _ptr(workspace),
                                 workspace.numel() * workspace.element_size(), _stream(stream)))


def dgemm_cublas(A, B, C, M, N, K, alpha=1.0, beta=0.0, stream=None) -> None:
    check(lib().lt_dgemm_cublas(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, _stream(stream)))


def dgemm_auto(A, B, C, M, N, K, alpha=1.0, beta=0.0, stream=None) -> tuple[int, int]:
    """lt_dgemm_auto: FP64-accurate DGEMM in the faster form; returns (form, slices) as chosen."""
    form, slices = ctypes.c_int(-1), ctypes.c_int(-1)
    check(lib().lt_dgemm_auto(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, ctypes.byref(form),
                              ctypes.byref(slices), _stream(stream)))
    return form.value, slices.value


def estimate_ms(form: int, M: int, N: int, K: int, slices: int = 0) -> float:
    """The auto form's cost model (host arithmetic only)."""
    return lib().lt_dgemm_estimate_ms(form, M, N, K, slices)


def ozaki_workspace_size(M, N, K, slices) -> int:
    return int(lib().lt_ozaki_workspace_size(M, N, K, slices))


def fill(X, n: int, seed: int, stream_id: int, phi: int = 0, stream=None) -> None:
    check(lib().lt_fill(_ptr(X), n, seed, stream_id, phi, _stream(stream)))


def scale_rows(X, rows, cols, seed, stream_id, smax, stream=None) -> None:
    check(lib().lt_scale_rows(_ptr(X), rows, cols, seed, stream_id, smax, _stream(stream)))


def scale_cols(X, rows, cols, seed, stream_id, smax, stream=None) -> None:
    check(lib().lt_scale_cols(_ptr(X), rows, cols, seed, stream_id, smax, _stream(stream)))


def device_status() -> None:
    check(lib().lt_check_device_status())


def fp64_configs() -> list[str]:
    L = lib()
    return [L.lt_fp64_config_name(i).decode() for i in range(L.lt_fp64_num_configs())]


def componentwise_error(C, Cref, den, n: int, tol: float = 0.0, stream=None) -> tuple[float, int]:
    out = (ctypes.c_double * 2)()
    check(lib().lt_componentwise_error(_ptr(C), _ptr(Cref), _ptr(den), n, tol, out, _stream(stream)))
    return float(out[0]), int(out[1])


def dot2_rows(A, B, C0, M, N, K, alpha, beta, rows, Cref, den, stream=None) -> None:
    """Compensated reference of the rows listed in the device int64 tensor `rows` (lt_dot2_rows):
    Cref and den are (len(rows), N) FP64 device tensors."""
    check(lib().lt_dot2_rows(_ptr(A), _ptr(B), _ptr(C0) if C0 is not None else None, alpha, beta, M, N, K, _ptr(rows),
                             int(rows.numel()), _ptr(Cref), _ptr(den), _stream(stream)))


def abs_denominator(A, B, C0, den, M, N, K, alpha, beta, stream=None) -> None:
    check(lib().lt_abs_denominator(_ptr(A), _ptr(B), None if C0 is None else _ptr(C0), _ptr(den), M, N, K,
                                   alpha, beta, _stream(stream)))


def measure_peak(kind: int, stream=None) -> float:
    """Measured rate (op/s, 2 per multiply-add) of one tensor instruction form on the current
    device: LT_PEAK_FP64_MMA, LT_PEAK_INT8_MMA_N128, LT_PEAK_INT8_MMA_N256 or LT_PEAK_INT8_MMA_PAIR."""
    out = ctypes.c_double()
    check(lib().lt_measure_peak(kind, ctypes.byref(out), _stream(stream)))
    return out.value


def dgemm_ozaki_host(A, B, C, M, N, K, alpha=1.0, beta=0.0, slices=8, stream=None) -> None:
    """Ozaki DGEMM on host (CPU) tensors or arrays, pipelined through the GPU (lt_dgemm_ozaki_host).
    C holds C0 on entry and the result on return."""
    check(lib().lt_dgemm_ozaki_host(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, slices, _stream(stream)))


def _half_bits(x: float) -> int:
    """IEEE binary16 bit pattern of x (round to nearest even)."""
    return int.from_bytes(struct.pack("<e", x), "little")


def hgemm(impl: str, A, B, C, M: int, N: int, K: int, alpha: float = 1.0, beta: float = 0.0) -> float:
    """Reference-contract call hgemm_<impl>(A, B, C, M, N, K, alpha, beta) on FP16 device tensors;
    returns the milliseconds the implementation measured (routines/hgemm/hgemm.h:6-7)."""
    fn = getattr(lib(), f"hgemm_{impl}")
    ms = fn(_ptr(A), _ptr(B), _ptr(C), M, N, K, _half_bits(alpha), _half_bits(beta))
    err = lib().lt_get_last_error()
    check(err)
    return ms


def hgemm_tc(A, B, C, M, N, K, alpha=1.0, beta=0.0, stream=None, config: int = -1) -> None:
    """C = alpha*A*B + beta*C on FP16 device tensors (lt_hgemm_config), FP32 accumulation."""
    check(lib().lt_hgemm_config(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, config, _stream(stream)))


def hgemm_cublas(A, B, C, M, N, K, alpha=1.0, beta=0.0, compute_f32: bool = True, stream=None) -> None:
    check(lib().lt_hgemm_cublas(_ptr(A), _ptr(B), _ptr(C), M, N, K, alpha, beta, int(compute_f32), _stream(stream)))


def hgemm_configs() -> list[str]:
    L = lib()
    return [L.lt_hgemm_config_name(i).decode() for i in range(L.lt_hgemm_num_configs())]


def dgemm_ex(transa: str, transb: str, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, form=LT_FORM_FP64, slices=8,
             stream=None) -> None:
    """BLAS-style DGEMM on row-major device matrices with row strides and transposes (lt_dgemm_ex)."""
    check(lib().lt_dgemm_ex(form, transa.encode(), transb.encode(), M, N, K, alpha, _ptr(A), lda, _ptr(B), ldb, beta,
                            _ptr(C), ldc, slices, _stream(stream)))
