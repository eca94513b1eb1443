"""CPU checks of the C ABI boundary: the library loads, exports every function declared in
include/*.h, and rejects bad arguments before touching a GPU."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"#[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("lt_", "dgemm_", "hgemm_")) and name not in names:
                names.append(name)
    return names


def test_header_declares_reference_contract():
    names = declared_functions()
    for impl in ["tc100", "cublas_tc", "ozaki_auto"] + [f"ozaki{s}" for s in range(3, 11)]:
        assert f"dgemm_{impl}" in names
    # the hgemm routine's contract (routines/hgemm/hgemm.h:6-7)
    assert "hgemm_tc100" in names and "hgemm_cublas" in names


def test_library_exports_every_declared_symbol():
    import libthom_b200 as lt

    L = lt.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    # and the Python layer knows every signature
    assert not [n for n in declared_functions() if n not in lt.SIGNATURES]


def test_errors_without_gpu():
    import libthom_b200 as lt

    L = lt.lib()
    assert L.lt_error_string(lt.LT_ERR_INVALID_ARGUMENT) == b"invalid argument"
    # argument validation happens before any device work
    rc = L.lt_dgemm_fp64(None, None, None, -1, 4, 4, 1.0, 0.0, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT and L.lt_get_last_error() == rc
    rc = L.lt_dgemm_ozaki(None, None, None, 4, 4, 4, 1.0, 0.0, 3, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT
    rc = L.lt_dgemm_ozaki(ctypes.c_void_p(0x1000), ctypes.c_void_p(0x1000), ctypes.c_void_p(0x1000), 4, 4, 4, 1.0,
                          0.0, 0, None)
    assert rc == lt.LT_ERR_INVALID_ARGUMENT  # slice count 0
    rc = L.lt_dgemm_fp64(ctypes.c_void_p(0x1004), ctypes.c_void_p(0x1000), ctypes.c_void_p(0x1000), 4, 4, 4, 1.0,
                         0.0, None)
    assert rc == lt.LT_ERR_UNALIGNED
    assert b"8-byte" in L.lt_last_error_message()
    assert L.lt_ozaki_workspace_size(8192, 8192, 8192, 8) >= 8 * 2 * 8192 * 8192
    assert L.lt_ozaki_workspace_size(8, 8, 8, 0) == 0
    assert L.lt_ozaki_analytic_slices(1e-15, 0) >= 8
    assert L.lt_ozaki_analytic_slices(-1.0, 0) == 0


def test_analytic_rule_matches_oracle(oracle_mod):
    import libthom_b200 as lt

    L = lt.lib()
    for tol in (1e-6, 1e-10, 1e-12, 1e-14, 1e-15):
        for gap in (0, 5, 20, 40, 64, 100):
            assert L.lt_ozaki_analytic_slices(tol, gap) == oracle_mod.analytic_slices(tol, gap)


def test_unknown_impl_rejected():
    import libthom_b200 as lt

    with pytest.raises(KeyError):
        lt.dgemm("final", 0, 0, 0, 1, 1, 1)


def test_dgemm_ex_rejects_bad_arguments():
    """Argument checks of lt_dgemm_ex run before any device work (no GPU needed)."""
    import libthom_b200 as lt

    L = lt.lib()
    ok_args = dict(M=4, N=4, K=4, lda=4, ldb=4, ldc=4)

    def call(form=lt.LT_FORM_FP64, ta=b"N", tb=b"N", slices=8, **kw):
        a = dict(ok_args, **kw)
        return L.lt_dgemm_ex(form, ta, tb, a["M"], a["N"], a["K"], 1.0, 8, a["lda"], 8, a["ldb"], 0.0, 8, a["ldc"],
                             slices, None)

    assert call(ta=b"X") == lt.LT_ERR_INVALID_ARGUMENT
    assert call(form=9) == lt.LT_ERR_INVALID_ARGUMENT
    assert call(form=lt.LT_FORM_OZAKI, slices=0) == lt.LT_ERR_INVALID_ARGUMENT
    assert call(lda=3) == lt.LT_ERR_INVALID_ARGUMENT
    assert call(ta=b"T", M=6, lda=5) == lt.LT_ERR_INVALID_ARGUMENT  # transposed A: lda >= M
    assert call(tb=b"T", K=6, ldb=5, lda=6) == lt.LT_ERR_INVALID_ARGUMENT  # transposed B: ldb >= K
    assert call(ldc=3) == lt.LT_ERR_INVALID_ARGUMENT
    assert call(M=-1) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dgemm_ex(0, b"N", b"N", 4, 4, 4, 1.0, 12, 4, 8, 4, 0.0, 8, 4, 8, None) == lt.LT_ERR_UNALIGNED


def test_hgemm_rejects_bad_arguments():
    """Argument checks of lt_hgemm run before any device work (no GPU needed)."""
    import libthom_b200 as lt

    L = lt.lib()
    p = ctypes.c_void_p(0x1000)
    assert L.lt_hgemm(p, p, p, -1, 4, 4, 1.0, 0.0, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_hgemm(None, p, p, 4, 4, 4, 1.0, 0.0, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_hgemm(ctypes.c_void_p(0x1001), p, p, 4, 4, 4, 1.0, 0.0, None) == lt.LT_ERR_UNALIGNED
    assert L.lt_hgemm_config(p, p, p, 4, 4, 4, 1.0, 0.0, 7, None) == lt.LT_ERR_NOT_FOUND
    assert L.lt_hgemm_num_configs() == len(lt.hgemm_configs()) >= 2
    # M == 0 or N == 0: nothing to do, no device touched
    assert L.lt_hgemm(p, p, p, 0, 4, 4, 1.0, 0.0, None) == lt.LT_OK


def test_dot2_rows_rejects_bad_arguments():
    """lt_dot2_rows validates before any device work (no GPU needed)."""
    import libthom_b200 as lt

    L = lt.lib()
    p = ctypes.c_void_p(0x1000)
    assert L.lt_dot2_rows(p, p, p, 1.0, 0.0, -1, 4, 4, p, 2, p, p, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dot2_rows(p, p, p, 1.0, 0.0, 4, 4, 4, None, 2, p, p, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dot2_rows(p, p, None, 1.0, 0.5, 4, 4, 4, p, 2, p, p, None) == lt.LT_ERR_INVALID_ARGUMENT  # C0 needed
    assert L.lt_dot2_rows(p, p, p, 1.0, 0.0, 4, 4, 4, p, 70000, p, p, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_dot2_rows(p, p, p, 1.0, 0.0, 4, 4, 4, p, 0, p, p, None) == lt.LT_OK  # nothing to do


def test_selftest_rejects_bad_limits_without_gpu():
    import libthom_b200 as lt

    L = lt.lib()
    for bad in (0.0, -1.0, 1e4, float("nan")):
        assert L.lt_selftest_wait_timeout(bad, None) == lt.LT_ERR_INVALID_ARGUMENT


def test_auto_form_cost_model_without_gpu():
    """lt_dgemm_estimate_ms is host arithmetic: the auto form's choices at the workload shapes."""
    import libthom_b200 as lt

    F, O = lt.LT_FORM_FP64, lt.LT_FORM_OZAKI
    # 8192^3 and K = 65536: the slice products win; 65536 x 64 x 4096 (the split of A dominates)
    # and small shapes: native FP64 wins even against 3 slices
    assert lt.estimate_ms(O, 8192, 8192, 8192, 7) < lt.estimate_ms(F, 8192, 8192, 8192) / 2.5
    assert lt.estimate_ms(O, 2048, 2048, 65536, 7) < lt.estimate_ms(F, 2048, 2048, 65536) / 2
    assert lt.estimate_ms(F, 65536, 64, 4096) < lt.estimate_ms(O, 65536, 64, 4096, 3)
    assert lt.estimate_ms(F, 512, 512, 512) < lt.estimate_ms(O, 512, 512, 512, 3)
    # 8192^3 FP64 at the measured 34.4 TF/s
    assert abs(lt.estimate_ms(F, 8192, 8192, 8192) - 2 * 8192 ** 3 / 34.4e9) < 0.1
    times = [lt.estimate_ms(O, 4096, 4096, 4096, s) for s in range(1, 13)]
    assert times == sorted(times)
    assert lt.estimate_ms(F, 0, 5, 5) == 0.0
    assert lt.estimate_ms(7, 8, 8, 8) == -1.0 and lt.estimate_ms(O, 8, 8, 8, 0) == -1.0
    assert lt.estimate_ms(O, 8, 8, 8, 13) == -1.0


def test_auto_plan_rejects_bad_arguments():
    """lt_ozaki_auto_plan_create checks its arguments before any device work; run/choice reject a
    missing plan and destroy accepts NULL."""
    import ctypes

    import libthom_b200 as lt

    L = lt.lib()
    h = ctypes.c_void_p()
    p = 0x1000
    bad = [
        (p, p, p, 0, 4, 4, 1e-12, lt.LT_AUTO_PLAN_OZAKI),       # empty
        (p, p, p, 4, 4, -1, 1e-12, lt.LT_AUTO_PLAN_OZAKI),      # negative K
        (None, p, p, 4, 4, 4, 1e-12, lt.LT_AUTO_PLAN_OZAKI),    # null A
        (p, p, p, 4, 4, 4, 0.0, lt.LT_AUTO_PLAN_OZAKI),         # no tolerance
        (p, p, p, 4, 4, 4, 1e-12, 7),                           # unknown forms
    ]
    for A, B, C, M, N, K, tol, forms in bad:
        assert L.lt_ozaki_auto_plan_create(A, B, C, M, N, K, 1.0, 0.0, tol, forms, ctypes.byref(h)) == \
            lt.LT_ERR_INVALID_ARGUMENT, (M, N, K, tol, forms)
        assert not h.value
    assert L.lt_ozaki_auto_plan_create(p + 4, p, p, 4, 4, 4, 1.0, 0.0, 1e-12, 0, ctypes.byref(h)) == lt.LT_ERR_UNALIGNED
    assert L.lt_ozaki_auto_plan_create(p, p, p, 4, 4, 4, 1.0, 0.0, 1e-12, 0, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_auto_plan_run(None, None) == lt.LT_ERR_INVALID_ARGUMENT
    assert L.lt_ozaki_auto_plan_choice(None, None, None) == lt.LT_ERR_INVALID_ARGUMENT
    L.lt_ozaki_auto_plan_destroy(None)
