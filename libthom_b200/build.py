"""Build recipe for the sm_100a DGEMM library and the libthom CLI.

Compiles every CUDA source under libthom_b200/csrc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) into the in-tree shared library
libthom_b200/liblibthom_dgemm.so, and the host harness under libthom_b200/host into
build/libthom (the reference's `./build/libthom test|bench|tune dgemm <impl> ...` entry point).
Objects are cached under libthom_b200/_build and rebuilt when a source or header is newer.

    python -m libthom_b200.build            # library + CLI
    python -m libthom_b200.build --lib      # library only
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
OBJ = PKG / "_build"
LIB = PKG / "liblibthom_dgemm.so"
CLI = ROOT / "build" / "libthom"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                     "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted((ROOT / "include").glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout)
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}")
    if os.environ.get("LT_BUILD_VERBOSE"):
        sys.stdout.write(res.stdout)


def _compile(src: Path, verbose_ptxas: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if _stale(obj, [src] + _headers()):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        _run(cmd)
    return obj


def build_library(jobs: int | None = None, verbose_ptxas: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), sources))
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] +
             ["-lcublas", "-Xlinker", "-rpath," + str(CUDA_HOME / "lib64")])
    return LIB


def build_cli() -> Path | None:
    sources = sorted(HOST.glob("*.cpp"))
    if not sources:
        return None
    CLI.parent.mkdir(exist_ok=True)
    deps = sources + sorted(HOST.glob("*.h")) + [LIB]
    if _stale(CLI, deps):
        _run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(HOST),
              "-I", str(CUDA_HOME / "include")] + [str(s) for s in sources] +
             ["-o", str(CLI), "-L", str(PKG), "-llibthom_dgemm", "-Wl,-rpath," + str(PKG),
              "-L", str(CUDA_HOME / "lib64"), "-lcudart", "-Wl,-rpath," + str(CUDA_HOME / "lib64"), "-lpthread"])
    return CLI


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", action="store_true", help="library only")
    ap.add_argument("--ptxas", action="store_true", help="print ptxas register/spill report")
    args = ap.parse_args()
    print(build_library(verbose_ptxas=args.ptxas))
    if not args.lib:
        print(build_cli())


if __name__ == "__main__":
    main()
