"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on the CPU.

The CPU oracle (oracle/) is the checker: it is built here on demand. The product library
(libthom_b200/liblibthom_dgemm.so) must already be built (python -m libthom_b200.build).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

U = 2.0 ** -53  # unit roundoff of binary64


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def golden():
    return np.load(ROOT / "tests" / "golden" / "dgemm_ref.npz")


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device and the loaded library; fails (not skips) if the library is absent."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import libthom_b200 as lt

    lt.lib()  # raises if the .so is missing: the product path has no fallback
    torch.cuda.init()
    return torch


def to_dev(torch, a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def fp64_bound(K: int) -> float:
    """Worst-case componentwise error of any FP64 dot-product order (with FMA) for length K,
    plus the alpha/beta epilogue roundings: (K + 4) u relative to |alpha||A||B| + |beta||C0|."""
    return (K + 4) * U


def tight_fp64_bound(e_cublas: float) -> float:
    """Statistical bar for the native FP64 kernels beside the worst case: for these inputs (random signs)
    the componentwise error of an FP64 product does not grow with K, so the kernel's error may be at
    most four times cuBLAS DGEMM's own on the same inputs, and at least 16 u where cuBLAS is nearly
    exact (tiny K)."""
    return max(4.0 * e_cublas, 16 * U)
