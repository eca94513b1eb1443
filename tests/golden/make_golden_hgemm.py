"""Generates tests/golden/hgemm_ref.npz from the reference's own HGEMM host check.

The loop is the reference's routines/hgemm/hgemm.cu:135-149 (hgemm::getReferenceResults),
compiled unmodified from the reference sources into oracle/_ref/libref_hgemm.so by oracle/Makefile.
Inputs are FP16 bit patterns from a seeded numpy generator (oracle.make_half_problem); the fixture
stores them with the reference's outputs, so the tests need neither the reference nor the generator.

    python tests/golden/make_golden_hgemm.py      # needs the reference sources to build oracle/_ref
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

# (M, N, K, alpha, beta, lo, hi): the reference runner's own setting (alpha 1, beta 0, uniform
# (0, 1), routines/hgemm/hgemm.cu:107-121), signed values with alpha/beta, K above one 64-wide block,
# tiny shapes, K = 1, results that overflow FP16 to Inf, and results in the FP16 subnormal range.
CASES = [
    (64, 64, 64, 1.0, 0.0, 0.0, 1.0),
    (17, 23, 31, 1.5, 0.5, -1.0, 1.0),
    (24, 40, 520, 1.0, 0.0, 0.0, 1.0),
    (1, 9, 3, 2.0, -1.0, -1.0, 1.0),
    (128, 8, 1, 1.0, 1.0, -1.0, 1.0),
    (16, 16, 160, 1.0, 0.0, 10.0, 30.0),
    (16, 24, 48, 0.5, 0.25, -1e-3, 1e-3),
]


def main() -> None:
    oracle.build()
    if oracle.ref_hgemm_lib() is None:
        raise SystemExit("oracle/_ref/libref_hgemm.so not built: the reference sources are needed")
    out = {}
    for i, (M, N, K, alpha, beta, lo, hi) in enumerate(CASES):
        A, B, C0 = oracle.make_half_problem(M, N, K, seed=1234 + i, lo=lo, hi=hi)
        ab, bb = int(oracle.half_bits(alpha)), int(oracle.half_bits(beta))
        C = oracle.hgemm_ref_loop(A, B, C0, ab, bb)
        out[f"case{i}_params"] = np.array([M, N, K], dtype=np.int64)
        out[f"case{i}_scalars"] = np.array([alpha, beta])
        out[f"case{i}_A"], out[f"case{i}_B"], out[f"case{i}_C0"], out[f"case{i}_C"] = A, B, C0, C
    out["ncases"] = np.array([len(CASES)])
    path = Path(__file__).with_name("hgemm_ref.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes, {len(CASES)} cases)")


if __name__ == "__main__":
    main()
