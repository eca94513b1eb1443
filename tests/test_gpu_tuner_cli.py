"""GPU tests of the single-problem FP64 autotuner and of the `libthom` command line.

lt_tune_fp64 validates every FP64 kernel configuration against cuBLAS FP64 before timing it (the
precedent is the reference's hgemm tuner, routines/hgemm/hgemm.cu:295-316) and records the fastest for
the shape class; afterwards lt_dgemm_fp64 picks it, so the tuned call must equal the forced
configuration bit for bit, and a table saved to a file and loaded in a fresh process must give the same
choice. The command line's `test dgemm <impl> M N K runs 1` checks every element against cuBLAS FP64
(componentwise, tolerance LIBTHOM_DGEMM_TOL = 1e-13): the [check] line must report none above it.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import to_dev

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "build" / "libthom"


@pytest.mark.parametrize("M,N,K", [(300, 200, 500), (1024, 1024, 1024)])
def test_tuner_choice_is_used_and_persists(cuda, oracle_mod, tmp_path, M, N, K):
    import libthom_b200 as lt

    torch = cuda
    L = lt.lib()
    best = lt.TuneEntry()
    lt.check(L.lt_tune_fp64(M, N, K, 3, ctypes.byref(best)))
    assert 0 <= best.config < L.lt_fp64_num_configs()
    assert best.ms > 0.0 and best.max_rel_err < 1e-8
    assert L.lt_tuner_lookup(M, N, K) == best.config
    # the tuned call (config -1) is the forced configuration, bit for bit
    A, B, C0 = oracle_mod.make_problem(M, N, K, phi=2, seed=M)
    dA, dB = to_dev(torch, A), to_dev(torch, B)
    c_tuned, c_forced = to_dev(torch, C0), to_dev(torch, C0)
    lt.dgemm_fp64(dA, dB, c_tuned, M, N, K, 1.5, 0.5)
    lt.dgemm_fp64(dA, dB, c_forced, M, N, K, 1.5, 0.5, config=best.config)
    torch.cuda.synchronize()
    lt.device_status()
    assert np.array_equal(c_tuned.cpu().numpy(), c_forced.cpu().numpy())
    # saved, then loaded by another process, the table gives the same choice
    path = tmp_path / "tune.txt"
    lt.check(L.lt_tuner_save(str(path).encode()))
    code = ("import sys; sys.path.insert(0, %r); import libthom_b200 as lt; L = lt.lib(); "
            "assert L.lt_tuner_load(%r) == 0; print(L.lt_tuner_lookup(%d, %d, %d))"
            % (str(ROOT), str(path).encode(), M, N, K))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert int(out.stdout.strip().splitlines()[-1]) == best.config


@pytest.mark.parametrize("impl", ["tc100", "ozaki7", "ozaki_crt15", "auto"])
def test_cli_test_command_checks_every_element(cuda, impl):
    assert CLI.exists()
    env = dict(os.environ, LIBTHOM_DGEMM_ALPHA="1.5", LIBTHOM_DGEMM_BETA="0.5")
    r = subprocess.run([str(CLI), "test", "dgemm", impl, "257", "129", "300", "2", "1"], capture_output=True,
                       text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    checks = re.findall(r"\[check\] max componentwise error vs cuBLAS FP64: (\S+) \((\d+) elements above", r.stdout)
    assert checks, r.stdout[-2000:]
    for err, above in checks:
        assert int(above) == 0 and float(err) < 1e-13, (impl, err, above)
    assert "# GFLOP/s:" in r.stdout


def test_cli_tune_command_saves_a_table(cuda, tmp_path):
    assert CLI.exists()
    path = tmp_path / "dgemm_fp64.txt"
    env = dict(os.environ, LIBTHOM_TUNE_FILE=str(path))
    r = subprocess.run([str(CLI), "tune", "dgemm", "384", "256", "640"], capture_output=True, text=True, timeout=300,
                       env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert re.search(r"\[best\] 384x256x640: \S+ ", r.stdout), r.stdout
    # one line per shape class, each dimension rounded up to a power of two: 512 256 1024
    assert any(line.startswith("512 256 1024 ") for line in path.read_text().splitlines()), path.read_text()


def test_cli_bench_writes_the_reference_csv(cuda, tmp_path):
    """`libthom bench dgemm <impl>` (the reference's bench_handler, routines/routines.h:132-169, with
    exportCSV, routines/dgemm/dgemm.cpp:209-219): one `M,N,K,gflops` row per bench size in
    bench_dgemm_<impl>.csv in the working directory, equal to the medians printed as
    `[size: n] ==> g`, and each GFLOP/s plausible for the form (2MNK / (ms 1e6), dgemm.cpp:161-165)."""
    assert CLI.exists()
    r = subprocess.run([str(CLI), "bench", "dgemm", "ozaki_crt14"], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    printed = {int(n): float(g) for n, g in re.findall(r"\[size: (\d+)\] ==> (\S+)", r.stdout)}
    lines = (tmp_path / "bench_dgemm_ozaki_crt14.csv").read_text().strip().splitlines()
    assert lines[0] == "M,N,K,gflops"
    rows = [line.split(",") for line in lines[1:]]
    assert len(rows) == len(printed) >= 3
    for M, N, K, g in rows:
        assert M == N == K and int(M) in printed
        assert abs(float(g) - printed[int(M)]) <= 1e-3 * printed[int(M)] + 1e-3
        assert 100.0 < float(g) < 400000.0, (M, g)  # 0.1 .. 400 TFLOP/s
    assert printed[max(printed)] > 50000.0, printed  # the largest size runs the CRT form above 50 TFLOP/s
