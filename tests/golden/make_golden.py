"""Generates tests/golden/dgemm_ref.npz from the reference's own host check loop.

The loop is the reference's routines/dgemm/dgemm.cpp:122-133 (dgemm::getReferenceResults),
compiled unmodified from the reference sources into oracle/_ref/libref_dgemm.so by
oracle/Makefile. Inputs come from the seeded generator (oracle.fill, identical on host and device),
so the fixture stores the generator parameters, a digest of the inputs, the first generator values
(pinning the generator itself) and the reference outputs.

    python tests/golden/make_golden.py      # needs the reference sources to build oracle/_ref
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402

# (M, N, K, alpha, beta, phi, smax): config 1 shape family, ragged shapes, alpha/beta of config 2,
# an exponent spread and the row/column scaling of config 4.
CASES = [
    (64, 64, 64, 1.0, 0.0, 0, 0),
    (17, 23, 31, 1.5, 0.5, 0, 0),
    (96, 40, 130, 1.5, 0.5, 8, 0),
    (33, 65, 200, -2.0, 0.25, 32, 0),
    (48, 24, 96, 1.0, 0.0, 0, 64),
    (1, 7, 5, 1.0, 1.0, 0, 0),
    (128, 128, 1, 1.0, 1.0, 0, 0),
]


def digest(*arrays: np.ndarray) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main() -> None:
    oracle.build()
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref/libref_dgemm.so not built: the reference sources are needed")
    out = {}
    for i, (M, N, K, alpha, beta, phi, smax) in enumerate(CASES):
        A, B, C0 = oracle.make_problem(M, N, K, phi=phi, seed=1234 + i, smax=smax)
        C = oracle.dgemm_ref(A, B, C0, alpha, beta)
        out[f"case{i}_params"] = np.array([M, N, K, phi, smax, 1234 + i], dtype=np.int64)
        out[f"case{i}_scalars"] = np.array([alpha, beta])
        out[f"case{i}_digest"] = np.frombuffer(digest(A, B, C0).encode(), dtype=np.uint8)
        out[f"case{i}_C"] = C
    # generator pin: first 16 values of streams 1..3 at seed 1234 with phi = 0, 8
    gen = [oracle.fill(1, 16, st, phi, 1234)[0] for st in (1, 2, 3) for phi in (0, 8)]
    out["generator_first16"] = np.stack(gen)
    out["ncases"] = np.array([len(CASES)])
    path = Path(__file__).with_name("dgemm_ref.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes, {len(CASES)} cases)")


if __name__ == "__main__":
    main()
