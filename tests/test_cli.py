"""CPU checks of the `libthom` command line (libthom_b200/host/): argv errors are handled like the
reference's `main.cpp` and `Handlers` (exit status 1, the same messages, the registry listed)
before any device work, so these run without a GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "build" / "libthom"

DGEMM_IMPLS = ({"tc100", "cublas_tc", "auto", "ozaki_auto"} | {f"ozaki{s}" for s in range(3, 11)}
               | {f"ozaki_crt{n}" for n in range(14, 19)})
HGEMM_IMPLS = {"tc100", "cublas"}


@pytest.fixture(scope="module")
def cli():
    if not CLI.exists():
        from libthom_b200 import build

        build.build_cli()
    assert CLI.exists(), "the libthom CLI did not build"
    return CLI


def run(cli, *args):
    r = subprocess.run([str(cli), *args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout, r.stderr


def listed(stderr: str) -> set[str]:
    line = next(ln for ln in stderr.splitlines() if ln.startswith("Available implementations:"))
    return set(line.split(":", 1)[1].split())


def test_too_few_parameters(cli):
    # main.cpp:48-51: fewer than 3 argv entries
    for args in [(), ("test",)]:
        rc, _, err = run(cli, *args)
        assert rc == 1
        assert err.startswith("Not enough parameters")


@pytest.mark.parametrize("args", [("run", "dgemm"), ("test", "sgemm"), ("bench", "nosuch")])
def test_unknown_mode_or_routine(cli, args):
    # main.cpp:56-64: both maps are looked up before the handler runs
    rc, _, err = run(cli, *args)
    assert rc == 1
    assert f"Invalid mode or routine: {args[0]} {args[1]}" in err
    assert "They must be registered in main.cpp" in err


@pytest.mark.parametrize("routine,impls", [("dgemm", DGEMM_IMPLS), ("hgemm", HGEMM_IMPLS)])
def test_missing_arguments_list_the_registry(cli, routine, impls):
    # routines.h:95-105 (test) and routines.h:136-144 (bench): usage, then the registry
    rc, _, err = run(cli, "test", routine)
    assert rc == 1
    assert "Missing arguments." in err
    assert f"Usage: ./libthom test {routine} <impl> <M> <N> <K> <nb_iter> <check_result=1>" in err
    assert listed(err) == impls
    rc, _, err = run(cli, "bench", routine)
    assert rc == 1
    assert f"Usage: ./libthom bench {routine} <impl>" in err
    assert listed(err) == impls


@pytest.mark.parametrize("routine,impls", [("dgemm", DGEMM_IMPLS), ("hgemm", HGEMM_IMPLS)])
@pytest.mark.parametrize("mode", ["test", "bench"])
def test_unknown_implementation(cli, routine, impls, mode):
    # routines.h:121-129 / 160-168: the registry lookup fails before any device work
    args = [mode, routine, "nosuch"] + (["64", "64", "64", "1"] if mode == "test" else [])
    rc, _, err = run(cli, *args)
    assert rc == 1
    assert "Invalid implementation. Either it doesnt exist, or it's not available for the ARCH" in err
    assert listed(err) == impls
    assert "CUDA error" not in err


@pytest.mark.parametrize("impl", ["nosuch", "ozaki", "ozakix", "ozaki0", "ozaki13", "fp64x"])
@pytest.mark.parametrize("mode", ["test", "bench"])
def test_batched_routine_rejects_unknown_implementation_before_device_work(cli, impl, mode):
    args = [mode, "dgemmb", impl] + (["8", "32", "64", "1"] if mode == "test" else [])
    rc, _, err = run(cli, *args)
    assert rc == 1
    assert f"Invalid implementation {impl}." in err
    assert "CUDA error" not in err


@pytest.mark.parametrize("args", [("test", "dgemmb"), ("test", "dgemmb", "fp64", "8", "32"),
                                  ("test", "dgemmb", "fp64", "0", "32", "64", "1"),
                                  ("test", "dgemmb", "fp64", "8", "64", "32", "1"),
                                  ("tune", "dgemmb", "x")])
def test_batched_routine_rejects_bad_sizes(cli, args):
    rc, _, err = run(cli, *args)
    assert rc == 1
    assert "CUDA error" not in err
    assert "Usage: ./libthom" in err or "bad arguments" in err
