"""The drop-in boundary proven from the reference's side.

oracle/ref_runner_shim.cpp compiles the reference's routines/dgemm/dgemm.cpp where it lies, with this
library's header: its static_asserts check at compile time that every exported dgemm_<impl> has the
reference's implementation type dgemm::DgemmImpl (dgemm.cpp:36), and its main() hands implementations
to the reference's own runner (dgemm::runner, dgemm.cpp:168-205) after dgemm_handler's set-up
(dgemm.cpp:228-231), with the runner's element-by-element check against its host loop switched on
(dgemm.cpp:137-159): that check prints "Number of different results" when any element differs.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
RUNNER = ROOT / "oracle" / "_ref" / "ref_runner"


def test_entry_points_have_the_reference_implementation_type():
    import oracle

    ref = Path(oracle.REFERENCE_SRC)
    if not (ref / "routines" / "dgemm" / "dgemm.cpp").exists():
        pytest.skip("reference sources absent")
    res = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", f"-I{ref}", f"-I{ref / 'routines'}",
                          f"-I{ROOT / 'include'}", "-I/usr/local/cuda/include",
                          str(ROOT / "oracle" / "ref_runner_shim.cpp")], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-2000:]


@pytest.mark.gpu
@pytest.mark.parametrize("impl,M,N,K", [("tc100", 512, 512, 512), ("ozaki7", 512, 512, 512),
                                        ("ozaki_crt15", 512, 512, 512), ("ozaki_crt15", 300, 260, 333),
                                        ("auto", 1024, 1024, 1024)])
def test_reference_runner_checks_our_implementations(cuda, impl, M, N, K):
    if not RUNNER.exists():
        pytest.skip("oracle/_ref/ref_runner not built (reference sources absent at build time)")
    res = subprocess.run([str(RUNNER), impl, str(M), str(N), str(K)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    assert "Number of different results" not in res.stdout, res.stdout[-2000:]
    assert f"[ref_runner] {impl} {M} {N} {K}:" in res.stdout
    assert "Kernel launch error" not in res.stderr
